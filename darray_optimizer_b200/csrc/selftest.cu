// Failure-path self-test: a kernel waits on an mbarrier phase that nothing completes (no thread arrives), with
// the same bounded-wait discipline as the pipeline kernels.  When the limit runs out it records DB200_ERR_TIMEOUT
// in the context's status word and returns, so the host sees the error at db200_synchronize and the context
// stays usable.  No fault, trap or hang is involved.
#include "internal.h"
#include "ptx.cuh"

namespace db200 {
namespace {

__global__ void wait_never_kernel(int* status, unsigned long long limit_ns) {
  __shared__ __align__(8) unsigned long long bar_storage;
  const uint32_t bar = smem_u32(&bar_storage);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbarrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long t0 = global_timer_ns();
    bool done = false;
    while (!done) {
      done = mbar_try_wait(bar, 0);  // phase 0 never completes: nobody arrives
      if (!done && global_timer_ns() - t0 > limit_ns) break;
    }
    if (!done) atomicExch(status, DB200_ERR_TIMEOUT);
    // complete the phase ourselves so the barrier is not left with a pending phase
    mbar_arrive(bar);
  }
  __syncthreads();
}

}  // namespace
}  // namespace db200

using namespace db200;

extern "C" int db200_selftest_wait_timeout(db200_context* ctx, int limit_ms) {
  if (!ctx) return DB200_ERR_INVALID;
  if (limit_ms < 1 || limit_ms > 5000) return fail(ctx, DB200_ERR_INVALID, "selftest: limit_ms out of [1, 5000]");
  wait_never_kernel<<<1, 32, 0, ctx->stream>>>(ctx->d_status, (unsigned long long)limit_ms * 1000000ull);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}
