// Failure-path self-test: a kernel waits on an mbarrier phase that nothing completes (no thread arrives), with
// the same bounded-wait discipline as the pipeline kernels.  When the limit runs out it records DB200_ERR_TIMEOUT
// in the context's status word and returns, so the host sees the error at db200_synchronize and the context
// stays usable.  No fault, trap or hang is involved.
#include "gridsync.cuh"
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

// The grid barrier of the cooperative LU panel with one CTA that never arrives: the others give up after
// limit_ns and report DB200_ERR_TIMEOUT.
__global__ void grid_barrier_never_kernel(unsigned* count, int* status, unsigned long long limit_ns) {
  grid_barrier(count, gridDim.x, status, DB200_ERR_TIMEOUT, limit_ns, blockIdx.x != 0);
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

extern "C" int db200_selftest_grid_barrier_timeout(db200_context* ctx, int limit_ms) {
  if (!ctx) return DB200_ERR_INVALID;
  if (limit_ms < 1 || limit_ms > 5000) return fail(ctx, DB200_ERR_INVALID, "selftest: limit_ms out of [1, 5000]");
  unsigned* count = static_cast<unsigned*>(slot_buffer(ctx, SLOT_SPARE, 256));
  if (!count) return DB200_ERR_NOMEM;
  DB200_CUDA(ctx, cudaMemsetAsync(count, 0, sizeof(unsigned), ctx->stream));
  int* status = ctx->d_status;
  unsigned long long limit = (unsigned long long)limit_ms * 1000000ull;
  void* args[] = {&count, &status, &limit};
  DB200_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)grid_barrier_never_kernel, dim3(4), dim3(64), args, 0,
                                              ctx->stream));
  count_launch(ctx);
  return DB200_OK;
}
