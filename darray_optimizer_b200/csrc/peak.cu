// FP64 throughput probes: the denominators of the FP64 kernels' roofline fractions.  The bf16 and HBM peaks come
// from measured cuBLAS / copy runs; FP64 has no such library figure here, so these kernels measure what the FP64
// pipes deliver on this GPU: back-to-back mma.sync.m16n8k8.f64 (the DMMA tiles of la64.cu and rbf64.cu) and
// back-to-back FP64 FMAs, each with eight independent accumulator chains per warp / thread, operands in
// registers, timed with CUDA events on the context's stream.
#include "internal.h"

namespace db200 {
namespace {

__device__ __forceinline__ void dmma_probe(double* d, const double* a, const double* b) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

__global__ void __launch_bounds__(256) dmma_peak_kernel(int iters, double* out) {
  double acc[8][4];
  double a[4], b[2];
  const double s = 1e-9 * (double)(threadIdx.x + 1);
#pragma unroll
  for (int e = 0; e < 4; ++e) a[e] = 1.0 + s * e;
  b[0] = 1.0 - s;
  b[1] = 1.0 + 2 * s;
#pragma unroll
  for (int c = 0; c < 8; ++c)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[c][e] = 0.0;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < 8; ++c) dmma_probe(acc[c], a, b);
  }
  double sum = 0.0;
#pragma unroll
  for (int c = 0; c < 8; ++c)
#pragma unroll
    for (int e = 0; e < 4; ++e) sum += acc[c][e];
  if (sum == 1.2345) out[0] = sum;  // never true: keeps the chains alive
}

__global__ void __launch_bounds__(256) dfma_peak_kernel(int iters, double* out) {
  double acc[8];
  const double x = 1.0 + 1e-9 * (double)threadIdx.x, y = 1.0 - 1e-12;
#pragma unroll
  for (int c = 0; c < 8; ++c) acc[c] = (double)c;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = fma(acc[c], y, x);
  }
  double sum = 0.0;
#pragma unroll
  for (int c = 0; c < 8; ++c) sum += acc[c];
  if (sum == 1.2345) out[0] = sum;
}

template <typename K>
int time_kernel(db200_context* ctx, K kernel, int blocks, int iters, double* out, float* ms) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  DB200_CUDA(ctx, cudaEventCreate(&e0));
  DB200_CUDA(ctx, cudaEventCreate(&e1));
  kernel<<<blocks, 256, 0, ctx->stream>>>(iters / 8, out);  // warm-up (clocks up, code loaded)
  count_launch(ctx);
  cudaEventRecord(e0, ctx->stream);
  kernel<<<blocks, 256, 0, ctx->stream>>>(iters, out);
  count_launch(ctx);
  cudaEventRecord(e1, ctx->stream);
  const cudaError_t e = cudaEventSynchronize(e1);
  if (e == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  DB200_CUDA(ctx, e);
  DB200_CUDA(ctx, cudaGetLastError());
  return DB200_OK;
}

}  // namespace
}  // namespace db200

using namespace db200;

extern "C" int db200_probe_fp64_peak(db200_context* ctx, double* dmma_tflops, double* dfma_tflops) {
  if (!ctx || !dmma_tflops || !dfma_tflops) return DB200_ERR_INVALID;
  double* out = static_cast<double*>(slot_buffer(ctx, SLOT_SPARE, 256));
  if (!out) return DB200_ERR_NOMEM;
  const int blocks = ctx->num_sms * 4;  // 32 warps per SM
  float ms = 0.f;
  // DMMA: 8 m16n8k8 per warp and iteration, 2 * 16 * 8 * 8 flops each
  const int it_mma = 20000;
  int st = time_kernel(ctx, dmma_peak_kernel, blocks, it_mma, out, &ms);
  if (st) return st;
  *dmma_tflops = (double)blocks * 8 * it_mma * 8 * 2048.0 / (ms * 1e-3) / 1e12;
  // DFMA: 8 FMAs per thread and iteration, 2 flops each
  const int it_fma = 400000;
  if ((st = time_kernel(ctx, dfma_peak_kernel, blocks, it_fma, out, &ms))) return st;
  *dfma_tflops = (double)blocks * 256 * it_fma * 8 * 2.0 / (ms * 1e-3) / 1e12;
  return DB200_OK;
}
