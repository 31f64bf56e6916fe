// FP64 device kernels of the log-barrier SVM dual solver (Newton step by Sherman-Morrison-Woodbury).
//
// Restates include/dbarrier.h:14-81 (f, gg, Grad_f, Grad_Phi, Grad, Hess_Phi) and the Newton / line-search
// arithmetic of tests/testsvm.cpp:243-321, with the Newton system solved as
//   (Z Z^T + diag(D)) s = -g   ->   (I + Z^T D^-1 Z) u = -Z^T D^-1 g,   s = -D^-1 (g + Z u)
// instead of the reference's PCG on (Z Z^T + D + n I) x = e_1 (include/dbarrier.h:84-139).
// Every pass over Z (n x r, column major, FP64) is HBM-bound: one thread per row i reads Z[i + k*ld] for
// k = 0..r-1, coalesced across the warp; r-vectors live in shared memory.
#include <cfloat>

#include "barrier.h"
#include "internal.h"

namespace db200 {
namespace {

constexpr int THREADS = 256;
constexpr int MAX_R_SMEM = 4096;  // r-vector staged in shared memory (32 KB)

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-reduce NV sums and atomically add them to out[0..NV).
template <int NV>
__device__ __forceinline__ void block_sum_add(double (&v)[NV], double* out) {
  __shared__ double red[NV][THREADS / 32];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    const double s = warp_sum(v[k]);
    if (lane == 0) red[k][warp] = s;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < THREADS / 32; ++w) s += red[threadIdx.x][w];
    atomicAdd(out + threadIdx.x, s);
  }
  __syncthreads();
}

// atomic max / min on non-negative doubles through their (monotone) bit patterns
__device__ __forceinline__ void atomic_max_pos(double* p, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_min_pos(double* p, double v) {
  atomicMin(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}

__device__ __forceinline__ double row_dot(const double* __restrict__ Z, long long ld, int i, int r,
                                          const double* s_vec) {
  double acc = 0.0;
  const double* zi = Z + i;
#pragma unroll 8
  for (int k = 0; k < r; ++k) acc = fma(zi[(long long)k * ld], s_vec[k], acc);
  return acc;
}

// Gradient and Hessian diagonal at a (Grad_f + Grad_Phi = Grad, Hess_Phi):
//   zw = Z (Z^T a),  g = zw - 1 + (-1/a + 1/(C - a))/t,  D = (1/a^2 + 1/(C - a)^2)/t,  dinv = 1/D
// Reductions into red[]: [0] sum(a), [1] sum(log a + log(C - a)), [2] max D, [3] min D.
__global__ void __launch_bounds__(THREADS) grad_hess_kernel(int n, int r, const double* __restrict__ Z, long long ld,
                                                            const double* __restrict__ w, const double* __restrict__ a,
                                                            double C, double t, double* __restrict__ g,
                                                            double* __restrict__ dinv, double* red,
                                                            const double* __restrict__ zw_in,
                                                            double* __restrict__ zw_out) {
  __shared__ double sw[MAX_R_SMEM];
  if (!zw_in)
    for (int k = threadIdx.x; k < r; k += blockDim.x) sw[k] = w[k];
  __syncthreads();
  double sums[2] = {0.0, 0.0};
  double dmax = 0.0, dmin = DBL_MAX;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ai = a[i], ci = C - ai;
    const double zw = zw_in ? zw_in[i] : row_dot(Z, ld, i, r, sw);
    if (zw_out) zw_out[i] = zw;
    g[i] = (zw - 1.0) + ((-1.0 / ai) + (1.0 / ci)) / t;
    const double D = ((1.0 / (ai * ai)) + (1.0 / (ci * ci))) / t;
    dinv[i] = 1.0 / D;
    sums[0] += ai;
    sums[1] += log(ai) + log(ci);
    dmax = fmax(dmax, D);
    dmin = fmin(dmin, D);
  }
  block_sum_add<2>(sums, red);
  // max / min through warp shuffles then one atomic per warp
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    dmin = fmin(dmin, __shfl_xor_sync(0xffffffffu, dmin, o));
  }
  if (threadIdx.x % 32 == 0) {
    atomic_max_pos(red + 2, dmax);
    atomic_min_pos(red + 3, dmin);
  }
}

// Newton direction from u:  s = -dinv * (g + Z u).  Reductions: [0] g.s, [1] sum(s), [2] max feasible step
// (min over i of -a/s for s < 0 and (C - a)/s for s > 0).
__global__ void __launch_bounds__(THREADS) direction_kernel(int n, int r, const double* __restrict__ Z, long long ld,
                                                            const double* __restrict__ u, const double* __restrict__ g,
                                                            const double* __restrict__ dinv,
                                                            const double* __restrict__ a, double C,
                                                            double* __restrict__ s, double* red) {
  __shared__ double su[MAX_R_SMEM];
  for (int k = threadIdx.x; k < r; k += blockDim.x) su[k] = u[k];
  __syncthreads();
  double sums[2] = {0.0, 0.0};
  double tmax = DBL_MAX;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double zu = row_dot(Z, ld, i, r, su);
    const double gi = g[i];
    const double si = -dinv[i] * (gi + zu);
    s[i] = si;
    sums[0] += gi * si;
    sums[1] += si;
    const double ai = a[i];
    if (si < 0.0) tmax = fmin(tmax, -ai / si);
    else if (si > 0.0) tmax = fmin(tmax, (C - ai) / si);
  }
  block_sum_add<2>(sums, red);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) tmax = fmin(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
  if (threadIdx.x % 32 == 0) atomic_min_pos(red + 2, tmax);
}

// out[k] = sum_i Z[i, k] * (scale_i * v_i)  (scale may be null): Z^T v, one block per group of columns,
// grid.y splits the rows.  FP64 atomics combine the row splits.
__global__ void __launch_bounds__(THREADS) gemv_t_kernel(int n, int r, const double* __restrict__ Z, long long ld,
                                                         const double* __restrict__ v, const double* __restrict__ scale,
                                                         double sign, double* out, int rows_per_split) {
  // 8 warps per block, each warp owns one column at a time; columns strided over blocks
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int r0 = blockIdx.y * rows_per_split;
  const int r1 = min(n, r0 + rows_per_split);
  for (int k = blockIdx.x * (THREADS / 32) + warp; k < r; k += gridDim.x * (THREADS / 32)) {
    const double* zk = Z + (long long)k * ld;
    double acc = 0.0;
    for (int i = r0 + lane; i < r1; i += 32) {
      const double vi = scale ? scale[i] * v[i] : v[i];
      acc = fma(zk[i], vi, acc);
    }
    acc = warp_sum(acc);
    if (lane == 0) atomicAdd(out + k, sign * acc);
  }
}

// Log-barrier sums at T candidate steps: out[k] = sum_i log(a_i + tau_k s_i) + log(C - a_i - tau_k s_i); a
// candidate that leaves the open box anywhere gets +inf in out[T + k] (infeasible count).
template <int T>
__global__ void __launch_bounds__(THREADS) linesearch_kernel(int n, const double* __restrict__ a,
                                                             const double* __restrict__ s, double C,
                                                             const double* __restrict__ taus, double* out) {
  double tau[T];
#pragma unroll
  for (int k = 0; k < T; ++k) tau[k] = taus[k];
  double sums[2 * T];
#pragma unroll
  for (int k = 0; k < 2 * T; ++k) sums[k] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ai = a[i], si = s[i];
#pragma unroll
    for (int k = 0; k < T; ++k) {
      const double x = fma(tau[k], si, ai), y = C - x;
      if (x > 0.0 && y > 0.0)
        sums[k] += log(x) + log(y);
      else
        sums[T + k] += 1.0;
    }
  }
  block_sum_add<2 * T>(sums, out);
}

// gradf = Z w - 1, gradphi = (-1/a + 1/(C-a))/t, grad = gradf + gradphi, D = (1/a^2 + 1/(C-a)^2)/t
// (include/dbarrier.h:48-81 one by one); red: [0] += sum a, [1] += sum(log a + log(C - a)).
__global__ void __launch_bounds__(THREADS) terms_kernel(int n, int r, const double* __restrict__ Z, long long ld,
                                                        const double* __restrict__ w, const double* __restrict__ a,
                                                        double C, double t, double* gf, double* gp, double* g,
                                                        double* D, double* red) {
  __shared__ double sw[MAX_R_SMEM];
  for (int k = threadIdx.x; k < r; k += blockDim.x) sw[k] = w[k];
  __syncthreads();
  double sums[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ai = a[i], ci = C - ai;
    const double f1 = row_dot(Z, ld, i, r, sw) - 1.0;
    const double p1 = ((-1.0 / ai) + (1.0 / ci)) / t;
    gf[i] = f1;
    gp[i] = p1;
    g[i] = f1 + p1;
    D[i] = ((1.0 / (ai * ai)) + (1.0 / (ci * ci))) / t;
    sums[0] += ai;
    sums[1] += log(ai) + log(ci);
  }
  block_sum_add<2>(sums, red);
}

// Negated residual of the Newton system (Z Z^T + D) s = -g:  res = g + Z v + s / dinv  with v = Z^T s.
// red: [0] += |res|^2, [1] += |g|^2.
__global__ void __launch_bounds__(THREADS) residual_kernel(int n, int r, const double* __restrict__ Z, long long ld,
                                                           const double* __restrict__ v, const double* __restrict__ g,
                                                           const double* __restrict__ dinv,
                                                           const double* __restrict__ s, double* __restrict__ res,
                                                           double* red, double* __restrict__ zv_out) {
  __shared__ double sv[MAX_R_SMEM];
  for (int k = threadIdx.x; k < r; k += blockDim.x) sv[k] = v[k];
  __syncthreads();
  double sums[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double gi = g[i];
    const double zv = row_dot(Z, ld, i, r, sv);
    if (zv_out) zv_out[i] = zv;
    const double ri = gi + zv + s[i] / dinv[i];
    res[i] = ri;
    sums[0] += ri * ri;
    sums[1] += gi * gi;
  }
  block_sum_add<2>(sums, red);
}

// Line-search inputs for a direction s: red [0] += g.s, [1] += sum s, [2] min feasible step (init DBL_MAX).
__global__ void __launch_bounds__(THREADS) step_stats_kernel(int n, const double* __restrict__ g,
                                                             const double* __restrict__ s,
                                                             const double* __restrict__ a, double C, double* red) {
  double sums[2] = {0.0, 0.0};
  double tmax = DBL_MAX;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double si = s[i], ai = a[i];
    sums[0] += g[i] * si;
    sums[1] += si;
    if (si < 0.0) tmax = fmin(tmax, -ai / si);
    else if (si > 0.0) tmax = fmin(tmax, (C - ai) / si);
  }
  block_sum_add<2>(sums, red);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) tmax = fmin(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
  if (threadIdx.x % 32 == 0) atomic_min_pos(red + 2, tmax);
}

__global__ void reciprocal_kernel(int n, const double* x, double* y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = 1.0 / x[i];
}

__global__ void vec_update_kernel(int n, double alpha, const double* x, double beta, double* y, double gamma) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = (x ? alpha * x[i] : 0.0) + (beta != 0.0 ? beta * y[i] : 0.0) + gamma;
}

__global__ void negate_kernel(int n, const double* x, double* y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = -x[i];
}

__global__ void axpy_kernel(int n, double alpha, const double* __restrict__ x, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = fma(alpha, x[i], y[i]);
}

// Primal value pieces at w = Z^T a:  sum_i max(0, 1 - (Z w)_i)
__global__ void __launch_bounds__(THREADS) hinge_kernel(int n, int r, const double* __restrict__ Z, long long ld,
                                                        const double* __restrict__ w, double* red,
                                                        const double* __restrict__ y, double b) {
  __shared__ double sw[MAX_R_SMEM];
  for (int k = threadIdx.x; k < r; k += blockDim.x) sw[k] = w[k];
  __syncthreads();
  double sums[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    sums[0] += fmax(0.0, 1.0 - row_dot(Z, ld, i, r, sw) - (y ? y[i] * b : 0.0));
  block_sum_add<1>(sums, red);
}

__global__ void scale_diag_kernel(double* M, int ldm, int r, double factor) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r; i += gridDim.x * blockDim.x) M[(long long)i * ldm + i] *= factor;
}

__global__ void add_identity_kernel(double* M, int ldm, int r) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r; i += gridDim.x * blockDim.x) M[(long long)i * ldm + i] += 1.0;
}

__global__ void init_red_kernel(double* red, int nsum, int nmax, int nmin) {
  const int i = threadIdx.x;
  if (i < nsum) red[i] = 0.0;
  else if (i < nsum + nmax) red[i] = 0.0;
  else if (i < nsum + nmax + nmin) red[i] = DBL_MAX;
}

// taus[k] = t0 beta^k (k < 16), t0 = min(1, 0.99 * *step_max), by repeated multiplication (the host forms the
// same values the same way)
__global__ void steps16_kernel(const double* step_max, double beta, double* taus) {
  if (threadIdx.x != 0) return;
  const double m = 0.99 * *step_max;
  double t = (m < 1.0) ? m : 1.0;  // as std::min(1.0, m): 1 when m is NaN
  for (int k = 0; k < 16; ++k) {
    taus[k] = t;
    t *= beta;
  }
}

__global__ void dot_kernel(int r, const double* x, const double* y, double* out) {
  double s = 0.0;
  for (int k = threadIdx.x; k < r; k += blockDim.x) s += x[k] * y[k];
  double v[1] = {s};
  block_sum_add<1>(v, out);
}

inline int rows_grid(db200_context* ctx, int n) {
  int b = (n + THREADS - 1) / THREADS;
  const int cap = 4 * ctx->num_sms;
  return b < 1 ? 1 : (b > cap ? cap : b);
}

}  // namespace

int bar_init_red(db200_context* ctx, double* red, int nsum, int nmax, int nmin) {
  init_red_kernel<<<1, 64, 0, ctx->stream>>>(red, nsum, nmax, nmin);
  count_launch(ctx);
  return cudaGetLastError() == cudaSuccess ? DB200_OK : cuda_fail(ctx, cudaGetLastError(), "init_red");
}

int bar_grad_hess(db200_context* ctx, int n, int r, const double* Z, long long ld, const double* w, const double* a,
                  double C, double t, double* g, double* dinv, double* red, const double* zw_in, double* zw_out) {
  if (r > MAX_R_SMEM) return fail(ctx, DB200_ERR_UNSUPPORTED, "barrier: rank > 4096");
  grad_hess_kernel<<<rows_grid(ctx, n), THREADS, 0, ctx->stream>>>(n, r, Z, ld, w, a, C, t, g, dinv, red, zw_in,
                                                                   zw_out);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_direction(db200_context* ctx, int n, int r, const double* Z, long long ld, const double* u, const double* g,
                  const double* dinv, const double* a, double C, double* s, double* red) {
  direction_kernel<<<rows_grid(ctx, n), THREADS, 0, ctx->stream>>>(n, r, Z, ld, u, g, dinv, a, C, s, red);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_gemv_t(db200_context* ctx, int n, int r, const double* Z, long long ld, const double* v, const double* scale,
               double sign, double* out) {
  DB200_CUDA(ctx, cudaMemsetAsync(out, 0, sizeof(double) * r, ctx->stream));
  const int col_blocks = (r + 7) / 8;
  int splits = (4 * ctx->num_sms + col_blocks - 1) / col_blocks;
  int rows = (n + splits - 1) / splits;
  rows = round_up(rows < 32 ? 32 : rows, 32);
  splits = (n + rows - 1) / rows;
  dim3 grid(col_blocks, splits);
  gemv_t_kernel<<<grid, THREADS, 0, ctx->stream>>>(n, r, Z, ld, v, scale, sign, out, rows);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_linesearch16(db200_context* ctx, int n, const double* a, const double* s, double C, const double* taus,
                     double* out) {
  DB200_CUDA(ctx, cudaMemsetAsync(out, 0, sizeof(double) * 32, ctx->stream));
  linesearch_kernel<16><<<rows_grid(ctx, n), THREADS, 0, ctx->stream>>>(n, a, s, C, taus, out);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_terms(db200_context* ctx, int n, int r, const double* Z, long long ld, const double* w, const double* a,
              double C, double t, double* gf, double* gp, double* g, double* D, double* red) {
  if (r > MAX_R_SMEM) return fail(ctx, DB200_ERR_UNSUPPORTED, "barrier: rank > 4096");
  terms_kernel<<<rows_grid(ctx, n), THREADS, 0, ctx->stream>>>(n, r, Z, ld, w, a, C, t, gf, gp, g, D, red);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_residual(db200_context* ctx, int n, int r, const double* Z, long long ld, const double* v, const double* g,
                 const double* dinv, const double* s, double* res, double* red, double* zv_out) {
  residual_kernel<<<rows_grid(ctx, n), THREADS, 0, ctx->stream>>>(n, r, Z, ld, v, g, dinv, s, res, red, zv_out);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_step_stats(db200_context* ctx, int n, const double* g, const double* s, const double* a, double C,
                   double* red) {
  step_stats_kernel<<<rows_grid(ctx, n), THREADS, 0, ctx->stream>>>(n, g, s, a, C, red);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_reciprocal(db200_context* ctx, int n, const double* x, double* y) {
  reciprocal_kernel<<<rows_grid(ctx, n), THREADS, 0, ctx->stream>>>(n, x, y);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_vec_update(db200_context* ctx, int n, double alpha, const double* x, double beta, double* y, double gamma) {
  vec_update_kernel<<<rows_grid(ctx, n), THREADS, 0, ctx->stream>>>(n, alpha, x, beta, y, gamma);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_negate(db200_context* ctx, int n, const double* x, double* y) {
  negate_kernel<<<rows_grid(ctx, n), THREADS, 0, ctx->stream>>>(n, x, y);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_axpy(db200_context* ctx, int n, double alpha, const double* x, double* y) {
  axpy_kernel<<<rows_grid(ctx, n), THREADS, 0, ctx->stream>>>(n, alpha, x, y);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_hinge(db200_context* ctx, int n, int r, const double* Z, long long ld, const double* w, double* red,
              const double* y, double b) {
  DB200_CUDA(ctx, cudaMemsetAsync(red, 0, sizeof(double), ctx->stream));
  hinge_kernel<<<rows_grid(ctx, n), THREADS, 0, ctx->stream>>>(n, r, Z, ld, w, red, y, b);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_add_identity(db200_context* ctx, double* M, int ldm, int r) {
  add_identity_kernel<<<(r + 255) / 256, 256, 0, ctx->stream>>>(M, ldm, r);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_scale_diag(db200_context* ctx, double* M, int ldm, int r, double factor) {
  scale_diag_kernel<<<(r + 255) / 256, 256, 0, ctx->stream>>>(M, ldm, r, factor);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_steps16(db200_context* ctx, const double* step_max, double beta, double* taus) {
  steps16_kernel<<<1, 32, 0, ctx->stream>>>(step_max, beta, taus);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int bar_dot(db200_context* ctx, int r, const double* x, const double* y, double* out) {
  DB200_CUDA(ctx, cudaMemsetAsync(out, 0, sizeof(double), ctx->stream));
  dot_kernel<<<1, THREADS, 0, ctx->stream>>>(r, x, y, out);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

}  // namespace db200
