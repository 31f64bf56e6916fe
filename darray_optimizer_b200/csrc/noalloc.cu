// Allocation-free variant of the fused RBF x sketch entry point.
//
// Some callers cannot allocate device memory: plugin hosts that hand out a stream but own every allocation
// (the library must not call cudaMalloc/cudaFree behind their allocator), code running under a strict
// memory budget, or a process that must not touch the allocator between set-up and a latency-critical phase.
// This entry point serves them.  Its scratch (packed split-fp16 points, norms and scales, packed Omega^T and the
// device status word) lives in one file-scope __device__ array of DB200_NOALLOC_SCRATCH_BYTES, which every GPU that
// loads the library holds until the process exits.  Nothing here calls cudaMalloc, cudaFree or any allocating
// library routine.
#include <cstdio>

#include "internal.h"

namespace db200 {
namespace {

// The scratch array.  In host code this name is only a host-side stand-in for the symbol; its device address
// must be obtained with cudaGetSymbolAddress on each device before a kernel may use it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[DB200_NOALLOC_SCRATCH_BYTES];

// Resolve the scratch array's device address in the current context.  Done on every call rather than cached per
// device: an address is only valid in the context it was resolved in, and a caller may make its own context
// current on the device, or reset the device, between calls.  The lookup costs microseconds against a call that
// waits for its kernels anyway.
int scratch_address(int device, void** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    std::fprintf(stderr, "db200_rbf_sketch_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", device,
                 cudaGetErrorString(e));
    return DB200_ERR_CUDA;
  }
  *out = p;
  return DB200_OK;
}

}  // namespace
}  // namespace db200

using namespace db200;

extern "C" int db200_rbf_sketch_noalloc(void* stream, int m, int n, int d, int l, const float* Xi, int ldxi,
                                        const float* Xj, int ldxj, int x_layout, const float* yi, const float* yj,
                                        const float* Omega, int ldo, float* Y, int ldy, float gamma) {
  if (m < 0 || n < 0 || d < 1 || l < 0) return DB200_ERR_INVALID;
  if (m == 0 || l == 0) return DB200_OK;
  if (d > 128) return DB200_ERR_UNSUPPORTED;
  if (!Y || ldy < m) return DB200_ERR_INVALID;
  if (n == 0) {
    // an empty sum: Y = 0, as db200_rbf_sketch gives (a memset allocates nothing)
    cudaStream_t st0 = static_cast<cudaStream_t>(stream);
    if (cudaMemset2DAsync(Y, sizeof(float) * (size_t)ldy, 0, sizeof(float) * (size_t)m, (size_t)l, st0) != cudaSuccess)
      return DB200_ERR_CUDA;
    return cudaStreamSynchronize(st0) == cudaSuccess ? DB200_OK : DB200_ERR_CUDA;
  }
  if (!Xi || !Xj || !Omega || ldo < n) return DB200_ERR_INVALID;
  if (x_layout == DB200_POINT_MAJOR) {
    if (ldxi < d || ldxj < d) return DB200_ERR_INVALID;
  } else if (x_layout == DB200_FEATURE_MAJOR) {
    if (ldxi < m || ldxj < n) return DB200_ERR_INVALID;
  } else {
    return DB200_ERR_INVALID;
  }

  // Scratch layout: [status | Xi packed | Xi norms | Xj packed | Xj norms | Omega^T packed | tile table],
  // 256-byte aligned.
  const int dp = feature_pad(d);
  const int mpad = point_pad(m), npad = point_pad(n);
  const bool same = (Xi == Xj && ldxi == ldxj && m == n);
  const SketchPlan plan = plan_sketch(l);
  size_t need = 256;
  need = align_up(need + (size_t)mpad * 2 * dp * 2, 256);
  need = align_up(need + packed_norm_floats(mpad) * 4, 256);
  if (!same) {
    need = align_up(need + (size_t)npad * 2 * dp * 2, 256);
    need = align_up(need + packed_norm_floats(npad) * 4, 256);
  }
  need = align_up(need + packed_sketch_halves(plan, npad) * 2, 256);
  need = align_up(need + tile_table_bytes(1), 256);
  if (need > (size_t)DB200_NOALLOC_SCRATCH_BYTES) {
    std::fprintf(stderr,
                 "db200_rbf_sketch_noalloc: m=%d n=%d d=%d l=%d needs %zu bytes of scratch, more than the fixed "
                 "%zu-byte array; use db200_rbf_sketch for this size\n",
                 m, n, d, l, need, (size_t)DB200_NOALLOC_SCRATCH_BYTES);
    return DB200_ERR_TOO_LARGE;
  }

  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return DB200_ERR_CUDA;
  void* base = nullptr;
  int st = scratch_address(device, &base);
  if (st) return st;

  // A context on the stack: it owns nothing and allocates nothing.
  db200_context ctx;
  ctx.device = device;
  ctx.stream = static_cast<cudaStream_t>(stream);
  if (cudaDeviceGetAttribute(&ctx.num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return DB200_ERR_CUDA;
  Carve carve{static_cast<char*>(base)};
  ctx.d_status = carve.take<int>(64);
  if (cudaMemsetAsync(ctx.d_status, 0, sizeof(int), ctx.stream) != cudaSuccess) return DB200_ERR_CUDA;

  PackedPoints pi, pj;
  void* xpi = carve.take<uint16_t>((size_t)mpad * 2 * dp);
  float* ni = carve.take<float>(packed_norm_floats(mpad));
  if ((st = pack_points(&ctx, Xi, ldxi, x_layout, m, d, dp, mpad, xpi, ni))) return st;
  pi.xp = xpi;
  pi.norms = ni;
  pi.n = m;
  pi.npad = mpad;
  pi.dp = dp;
  if (same) {
    pj = pi;
  } else {
    void* xpj = carve.take<uint16_t>((size_t)npad * 2 * dp);
    float* nj = carve.take<float>(packed_norm_floats(npad));
    if ((st = pack_points(&ctx, Xj, ldxj, x_layout, n, d, dp, npad, xpj, nj))) return st;
    pj.xp = xpj;
    pj.norms = nj;
    pj.n = n;
    pj.npad = npad;
    pj.dp = dp;
  }
  void* op = carve.take<uint16_t>(packed_sketch_halves(plan, npad));
  if ((st = pack_sketch(&ctx, Omega, ldo, yj, n, l, npad, plan.lrows, op))) return st;
  void* table = carve.take<char>(tile_table_bytes(1));  // the tile engine's one-instance table
  if ((st = launch_rbf_tiles(&ctx, RBF_MODE_SKETCH, pi, pj, yi, nullptr, op, plan, l, gamma, Y, ldy, table,
                             tile_table_bytes(1))))
    return st;

  // Synchronous: wait, then report a device-side wait that gave up.
  // The status read is ordered on the caller's stream only: a cudaMemcpy on the legacy default stream would also
  // wait for every other blocking stream of the process.
  int dev_status = 0;
  if (cudaMemcpyAsync(&dev_status, ctx.d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream) != cudaSuccess)
    return DB200_ERR_CUDA;
  if (cudaStreamSynchronize(ctx.stream) != cudaSuccess) return DB200_ERR_CUDA;
  return dev_status;
}
