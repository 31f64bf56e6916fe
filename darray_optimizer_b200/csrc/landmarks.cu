// Learned Nystrom landmarks: k-NN distance features, the leverage MLP (forward, backward, Adam, all hand-written
// kernels), Gumbel top-k selection, the landmark Nystrom factor, a sampled residual estimate and ridge leverage
// scores from a low-rank factor.
//
// The reference always sketches with a Gaussian test matrix (include/dkernel.h:13-46, tests/testsvm.cpp:94-134);
// this file replaces Omega by r landmark columns of K when a model of the ridge leverage scores picks landmarks
// whose Nystrom factor meets a residual tolerance.  The factor is the column form of the Nystrom approximation,
// K ~ K(:, L) K(L, L)^-1 K(L, :), with the same y-folding as the sketch (Q = diag(y) K diag(y), dkernel.cu:125).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include <cuda_bf16.h>

#include "internal.h"
#include "la64.h"

struct db200_mlp {
  int in = 0, width = 0, hidden = 0, layers = 0, nparams = 0, device = 0;
  float* master = nullptr;        // fp32 parameters
  float* grad = nullptr;          // fp32 gradient of the last call
  float* mom1 = nullptr;          // Adam first moment
  float* mom2 = nullptr;          // Adam second moment
  __nv_bfloat16* wbf = nullptr;   // bf16 copy of the parameters used by the forward and backward passes
  float* in_mean = nullptr;
  float* in_scale = nullptr;
  double* d_loss = nullptr;
  long long step = 0;
  void* act = nullptr;            // activations / backward buffers, grow-only
  size_t act_bytes = 0;
  std::vector<int> off_w, off_b, fan_in, fan_out;
};

namespace db200 {

namespace {

inline unsigned blocks_for(long long total, int threads, long long cap = 65535LL * 16) {
  long long b = (total + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (unsigned)b;
}

// ------------------------------------------------------------------ k-NN distance
// One thread per query point, the query in registers (DMAX >= d), reference points staged through shared memory
// 64 at a time; the k smallest squared distances are kept sorted in registers.
constexpr int KNN_THREADS = 128, KNN_TILE = 64, KNN_KMAX = 16;

template <int DMAX>
__global__ void __launch_bounds__(KNN_THREADS) knn_kernel(int n, int d, const float* __restrict__ X, int ldx, int s,
                                                          const int* __restrict__ ref, int k, float* __restrict__ out) {
  __shared__ float sR[KNN_TILE][DMAX + 1];
  __shared__ int sI[KNN_TILE];
  const int i = blockIdx.x * KNN_THREADS + threadIdx.x;
  float q[DMAX];
#pragma unroll
  for (int c = 0; c < DMAX; ++c) q[c] = (i < n && c < d) ? X[(long long)i * ldx + c] : 0.f;
  float best[KNN_KMAX];
#pragma unroll
  for (int t = 0; t < KNN_KMAX; ++t) best[t] = INFINITY;
  for (int t0 = 0; t0 < s; t0 += KNN_TILE) {
    __syncthreads();
    for (int e = threadIdx.x; e < KNN_TILE * DMAX; e += KNN_THREADS) {
      const int jj = e / DMAX, c = e % DMAX;
      const int j = t0 + jj;
      sR[jj][c] = (j < s && c < d) ? X[(long long)ref[j] * ldx + c] : 0.f;
    }
    if (threadIdx.x < KNN_TILE) sI[threadIdx.x] = (t0 + threadIdx.x < s) ? ref[t0 + threadIdx.x] : -1;
    __syncthreads();
    const int cnt = min(KNN_TILE, s - t0);
    for (int jj = 0; jj < cnt; ++jj) {
      float dist = 0.f;
#pragma unroll
      for (int c = 0; c < DMAX; ++c) {
        const float df = q[c] - sR[jj][c];
        dist = fmaf(df, df, dist);
      }
      if (sI[jj] == i) continue;  // a point is not its own neighbour
      if (dist < best[KNN_KMAX - 1]) {
        // insertion into the sorted list (only the first k entries are used)
#pragma unroll
        for (int t = KNN_KMAX - 1; t > 0; --t) {
          const bool shift = dist < best[t - 1];
          best[t] = shift ? best[t - 1] : (dist < best[t] ? dist : best[t]);
        }
        if (dist < best[0]) best[0] = dist;
      }
    }
  }
  if (i < n) {
    float v = best[0];
#pragma unroll
    for (int t = 0; t < KNN_KMAX; ++t)
      if (t == k - 1) v = best[t];
    out[i] = sqrtf(v);
  }
}

// Rows ref[j] of X (point-major) gathered into R (s x d, point-major with leading dimension d).
__global__ void gather_rows_kernel(const float* __restrict__ X, int ldx, const int* __restrict__ ref, int s, int d,
                                   float* __restrict__ R) {
  const long long total = (long long)s * d;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(e / d), c = (int)(e % d);
    R[e] = X[(long long)ref[j] * ldx + c];
  }
}

// out[i] = sqrt of the k-th smallest of the 32 candidates part[32 i ..] (four sorted quarters of 8).
__global__ void knn_merge_kernel(int n, const float* __restrict__ part, int k, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float best[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) best[t] = INFINITY;
  const float* p = part + (size_t)i * 32;
#pragma unroll 4
  for (int c = 0; c < 32; ++c) {
    float x = p[c];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const float lo = fminf(best[t], x), hi = fmaxf(best[t], x);
      best[t] = lo;
      x = hi;
    }
  }
  float v = best[0];
#pragma unroll
  for (int t = 0; t < 8; ++t)
    if (t == k - 1) v = best[t];
  out[i] = sqrtf(fmaxf(v, 0.0f));
}


// F[i, :] = [x_i (d), ||x_i||, knn_i], row major n x (d + 2); one warp per point.
__global__ void features_kernel(int n, int d, const float* __restrict__ X, int ldx, const float* __restrict__ knn,
                                float* __restrict__ F) {
  const int lane = threadIdx.x % 32;
  const long long warps = (long long)gridDim.x * (blockDim.x / 32);
  for (long long i = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; i < n; i += warps) {
    float ss = 0.f;
    float* row = F + i * (d + 2);
    for (int c = lane; c < d; c += 32) {
      const float x = X[i * ldx + c];
      row[c] = x;
      ss = fmaf(x, x, ss);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if (lane == 0) {
      row[d] = sqrtf(ss);
      row[d + 1] = knn[i];
    }
  }
}

// lev_i = sum_c W(i, c)^2, W n x r column major (FP64)
__global__ void row_sumsq64_kernel(int n, int r, const double* __restrict__ W, long long ldw, double* __restrict__ lev) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int c = 0; c < r; ++c) {
      const double v = W[(long long)c * ldw + i];
      s = fma(v, v, s);
    }
    lev[i] = s;
  }
}

// ------------------------------------------------------------------ gathers
__global__ void gather_rows_f32_kernel(const float* __restrict__ X, int ldx, const int* __restrict__ idx, int r, int d,
                                       float* __restrict__ out) {
  const long long total = (long long)r * d;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(e / d), c = (int)(e % d);
    out[e] = X[(long long)idx[a] * ldx + c];
  }
}
__global__ void gather_f32_kernel(const float* __restrict__ v, const int* __restrict__ idx, int r, float* __restrict__ out) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < r; a += gridDim.x * blockDim.x) out[a] = v[idx[a]];
}
// out(a, b) = M(idx[a], b), M column major (ldm) with `cols` columns, out column major r x cols (ld r)
template <typename TS>
__global__ void gather_matrix_rows_kernel(const TS* __restrict__ M, long long ldm, const int* __restrict__ idx, int r,
                                          int cols, double* __restrict__ out) {
  const long long total = (long long)r * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(e % r), b = (int)(e / r);
    out[e] = (double)M[(long long)b * ldm + idx[a]];
  }
}

// ------------------------------------------------------------------ Gumbel keys and radix selection
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  // splitmix64 finaliser (Vigna): a bijective avalanche mix of a 64-bit counter
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__global__ void gumbel_kernel(int n, const float* __restrict__ logits, unsigned long long seed, float* __restrict__ keys) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned long long h = mix64(seed * 0x9e3779b97f4a7c15ull + (unsigned long long)i + 1ull);
    // uniform in (0, 1) from the top 53 bits
    const double u = ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    keys[i] = logits[i] + (float)(-log(-log(u)));
  }
}
__device__ __forceinline__ unsigned int key_bits(float f) {
  const unsigned int b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);  // order preserving: larger float -> larger unsigned
}
// histogram of byte `shift` of the keys whose higher bytes equal `prefix` (under `mask`)
__global__ void radix_hist_kernel(int n, const float* __restrict__ keys, unsigned int prefix, unsigned int mask, int shift,
                                  unsigned int* __restrict__ hist) {
  __shared__ unsigned int h[256];
  for (int b = threadIdx.x; b < 256; b += blockDim.x) h[b] = 0;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned int u = key_bits(keys[i]);
    if ((u & mask) == prefix) atomicAdd(&h[(u >> shift) & 0xFFu], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < 256; b += blockDim.x)
    if (h[b]) atomicAdd(&hist[b], h[b]);
}
// indices with key > thr, and the first `ties` (by arrival) with key == thr
__global__ void radix_compact_kernel(int n, const float* __restrict__ keys, unsigned int thr, int ties,
                                     unsigned int* __restrict__ counters, int* __restrict__ idx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned int u = key_bits(keys[i]);
    if (u > thr) {
      idx[atomicAdd(&counters[0], 1u)] = i;
    } else if (u == thr) {
      const unsigned int t = atomicAdd(&counters[1], 1u);
      if ((int)t < ties) idx[atomicAdd(&counters[0], 1u)] = i;
    }
  }
}

// ------------------------------------------------------------------ MLP
// C(i, j) = sum_k A(i, k) B(k, j), A(i, k) = A[i*a_i + k*a_k], B(k, j) = B[k*b_k + j*b_j], 64 x 64 tiles, 16-deep
// stages, 256 threads with 4 x 4 outputs each, fp32 accumulation.  grid.z splits K (EPI_ATOMIC only).
enum { EPI_HIDDEN = 0, EPI_OUT = 1, EPI_DH = 2, EPI_ATOMIC = 3 };
constexpr int MT = 64, MK = 16;

template <typename T>
__device__ __forceinline__ float tof(T v) { return (float)v; }
template <>
__device__ __forceinline__ float tof<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename TA, typename TB, int EPI>
__global__ void __launch_bounds__(256) mlp_gemm_kernel(int M, int N, int K, const TA* __restrict__ A, long long a_i,
                                                       long long a_k, const TB* __restrict__ B, long long b_k,
                                                       long long b_j, const float* __restrict__ bias,
                                                       const __nv_bfloat16* __restrict__ H, long long ldh, void* Cv,
                                                       long long ldc, int k_per_split) {
  __shared__ float sA[MK][MT + 1];
  __shared__ float sB[MK][MT + 1];
  const int i0 = blockIdx.x * MT, j0 = blockIdx.y * MT;
  const int kb = blockIdx.z * k_per_split, ke = min(K, kb + k_per_split);
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  float acc[4][4] = {};
  for (int k0 = kb; k0 < ke; k0 += MK) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int e = threadIdx.x + 256 * s;
      // walk the unit-stride index fastest for coalesced loads
      int ii, kk;
      if (a_k == 1) { kk = e % MK; ii = e / MK; } else { ii = e % MT; kk = e / MT; }
      const int gi = i0 + ii, gk = k0 + kk;
      sA[kk][ii] = (gi < M && gk < ke) ? tof(A[gi * a_i + gk * a_k]) : 0.f;
      int jj, kk2;
      if (b_k == 1) { kk2 = e % MK; jj = e / MK; } else { jj = e % MT; kk2 = e / MT; }
      const int gj = j0 + jj, gk2 = k0 + kk2;
      sB[kk2][jj] = (gj < N && gk2 < ke) ? tof(B[gk2 * b_k + gj * b_j]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < MK; ++t) {
      float av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = sA[t][ty * 4 + a];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = sB[t][tx * 4 + b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fmaf(av[a], bv[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = i0 + ty * 4 + a;
    if (i >= M) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int j = j0 + tx * 4 + b;
      if (j >= N) continue;
      const float v = acc[a][b];
      if (EPI == EPI_HIDDEN) {
        static_cast<__nv_bfloat16*>(Cv)[i * ldc + j] = __float2bfloat16_rn(fmaxf(v + bias[j], 0.f));
      } else if (EPI == EPI_OUT) {
        static_cast<float*>(Cv)[i * ldc + j] = v + bias[j];
      } else if (EPI == EPI_DH) {
        static_cast<float*>(Cv)[i * ldc + j] = (__bfloat162float(H[i * ldh + j]) > 0.f) ? v : 0.f;
      } else {
        atomicAdd(static_cast<float*>(Cv) + i * ldc + j, v);
      }
    }
  }
}

__global__ void standardize_kernel(int m, int in, const float* __restrict__ F, const float* __restrict__ mean,
                                   const float* __restrict__ scale, __nv_bfloat16* __restrict__ H0) {
  const long long total = (long long)m * in;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % in);
    H0[e] = __float2bfloat16_rn((F[e] - mean[c]) * scale[c]);
  }
}
// dout = (out - t) / m, loss += 0.5 (out - t)^2 / m
__global__ void mse_kernel(int m, const float* __restrict__ out, const float* __restrict__ t, float* __restrict__ dout,
                           double* loss) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const float r = out[i] - t[i];
    dout[i] = r / (float)m;
    s += 0.5 * (double)r * (double)r / (double)m;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x % 32 == 0) atomicAdd(loss, s);
}
// g[j] += sum_i dY[i*N + j]
__global__ void colsum_kernel(int m, int N, const float* __restrict__ dY, float* __restrict__ g) {
  const int j = blockIdx.x * 32 + threadIdx.x % 32;
  if (j >= N) return;
  float s = 0.f;
  for (int i = blockIdx.y * (blockDim.x / 32) + threadIdx.x / 32; i < m; i += gridDim.y * (blockDim.x / 32))
    s += dY[(long long)i * N + j];
  atomicAdd(g + j, s);
}
__global__ void adam_kernel(int np, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, __nv_bfloat16* __restrict__ wbf, float lr, float c1, float c2) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < np; e += gridDim.x * blockDim.x) {
    const float gi = g[e];
    const float a = 0.9f * m1[e] + 0.1f * gi;
    const float b = 0.999f * m2[e] + 0.001f * gi * gi;
    m1[e] = a;
    m2[e] = b;
    const float v = w[e] - lr * (a * c1) / (sqrtf(b * c2) + 1e-8f);
    w[e] = v;
    wbf[e] = __float2bfloat16_rn(v);
  }
}
__global__ void to_bf16_kernel(int np, const float* __restrict__ w, __nv_bfloat16* __restrict__ wbf) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < np; e += gridDim.x * blockDim.x) wbf[e] = __float2bfloat16_rn(w[e]);
}

template <typename TA, typename TB, int EPI>
int mlp_gemm(db200_context* ctx, int M, int N, int K, const TA* A, long long a_i, long long a_k, const TB* B,
             long long b_k, long long b_j, const float* bias, const __nv_bfloat16* H, long long ldh, void* C,
             long long ldc, int splits = 1) {
  if (M <= 0 || N <= 0) return DB200_OK;
  int kps = (K + splits - 1) / splits;
  kps = round_up(kps < MK ? MK : kps, MK);
  splits = (K + kps - 1) / kps;
  dim3 grid((M + MT - 1) / MT, (N + MT - 1) / MT, splits < 1 ? 1 : splits);
  if (grid.y > 65535 || grid.z > 65535) return fail(ctx, DB200_ERR_UNSUPPORTED, "mlp: GEMM too large");
  mlp_gemm_kernel<TA, TB, EPI><<<grid, 256, 0, ctx->stream>>>(M, N, K, A, a_i, a_k, B, b_k, b_j, bias, H, ldh, C,
                                                             ldc, kps);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

// activation buffers of one forward/backward over m rows
struct MlpActs {
  __nv_bfloat16* h[8];  // h[0] = standardised input (m x in), h[l] = layer l output (m x width), l = 1..hidden
  float* out;           // m
  float* dy0;           // m x max(width, 1)
  float* dy1;
};

int mlp_acts(db200_context* ctx, db200_mlp* net, int m, MlpActs* A) {
  const size_t hb = align_up((size_t)m * std::max(net->in, net->width) * 2, 256);
  const size_t need = (size_t)(net->hidden + 1) * hb + align_up((size_t)m * 4, 256) +
                      2 * align_up((size_t)m * net->width * 4, 256) + 1024;
  if (need > net->act_bytes) {
    DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (net->act) cudaFree(net->act);
    net->act = nullptr;
    net->act_bytes = 0;
    DB200_CUDA(ctx, cudaMalloc(&net->act, need));
    net->act_bytes = need;
  }
  Carve cv{static_cast<char*>(net->act)};
  for (int l = 0; l <= net->hidden; ++l) A->h[l] = reinterpret_cast<__nv_bfloat16*>(cv.take<char>(hb));
  A->out = cv.take<float>(m);
  A->dy0 = cv.take<float>((size_t)m * net->width);
  A->dy1 = cv.take<float>((size_t)m * net->width);
  return DB200_OK;
}

int mlp_forward_impl(db200_context* ctx, db200_mlp* net, int m, const float* F, MlpActs& A) {
  standardize_kernel<<<blocks_for((long long)m * net->in, 256), 256, 0, ctx->stream>>>(m, net->in, F, net->in_mean,
                                                                                         net->in_scale, A.h[0]);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  int st;
  for (int l = 0; l < net->layers; ++l) {
    const int K = net->fan_in[l], N = net->fan_out[l];
    const __nv_bfloat16* W = net->wbf + net->off_w[l];
    const float* b = net->master + net->off_b[l];
    if (l < net->hidden)
      st = mlp_gemm<__nv_bfloat16, __nv_bfloat16, EPI_HIDDEN>(ctx, m, N, K, A.h[l], K, 1, W, 1, K, b, nullptr, 0,
                                                             A.h[l + 1], N);
    else
      st = mlp_gemm<__nv_bfloat16, __nv_bfloat16, EPI_OUT>(ctx, m, N, K, A.h[l], K, 1, W, 1, K, b, nullptr, 0,
                                                          A.out, N);
    if (st) return st;
  }
  return DB200_OK;
}

// gradient of 0.5 mean (out - t)^2 into net->grad; loss into net->d_loss
int mlp_backward_impl(db200_context* ctx, db200_mlp* net, int m, const float* target, MlpActs& A) {
  DB200_CUDA(ctx, cudaMemsetAsync(net->grad, 0, sizeof(float) * net->nparams, ctx->stream));
  DB200_CUDA(ctx, cudaMemsetAsync(net->d_loss, 0, sizeof(double), ctx->stream));
  mse_kernel<<<blocks_for(m, 256, 1024), 256, 0, ctx->stream>>>(m, A.out, target, A.dy0, net->d_loss);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  float* dY = A.dy0;  // gradient at the output of layer l (m x fan_out[l])
  float* dX = A.dy1;
  const int splits = std::max(1, std::min(64, m / 512));
  int st;
  for (int l = net->layers - 1; l >= 0; --l) {
    const int K = net->fan_in[l], N = net->fan_out[l];
    // dW_l (N x K) = dY^T H_l  (sum over the m rows, split with atomics)
    if ((st = mlp_gemm<float, __nv_bfloat16, EPI_ATOMIC>(ctx, N, K, m, dY, 1, N, A.h[l], K, 1, nullptr, nullptr, 0,
                                                         net->grad + net->off_w[l], K, splits)))
      return st;
    colsum_kernel<<<dim3((N + 31) / 32, std::max(1, std::min(256, m / 256))), 256, 0, ctx->stream>>>(
        m, N, dY, net->grad + net->off_b[l]);
    DB200_CUDA(ctx, cudaGetLastError());
    count_launch(ctx);
    if (l > 0) {
      // dH_{l-1} (m x K) = (dY W_l) masked by ReLU'(H_{l-1})
      if ((st = mlp_gemm<float, __nv_bfloat16, EPI_DH>(ctx, m, K, N, dY, N, 1, net->wbf + net->off_w[l], K, 1,
                                                      nullptr, A.h[l], K, dX, K)))
        return st;
      std::swap(dY, dX);
    }
  }
  return DB200_OK;
}

// Uniform sample of s distinct indices of [0, n) (partial Fisher-Yates, seeded), sorted.
std::vector<int> sample_indices(int n, int s, unsigned long long seed) {
  s = std::min(s, n);
  std::vector<int> p(n);
  for (int i = 0; i < n; ++i) p[i] = i;
  std::mt19937_64 g(seed);
  for (int i = 0; i < s; ++i) {
    std::uniform_int_distribution<int> u(i, n - 1);
    std::swap(p[i], p[u(g)]);
  }
  p.resize(s);
  std::sort(p.begin(), p.end());
  return p;
}

struct LandTimer {
  cudaStream_t s;
  cudaEvent_t a = nullptr, b = nullptr;
  explicit LandTimer(cudaStream_t st) : s(st) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
  }
  double stop() {
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
  ~LandTimer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

}  // namespace

// ------------------------------------------------------------------ internal entry points (shared with C ABI)
int knn_distance(db200_context* ctx, int n, int d, const float* X, int ldx, int s, const int* ref, int k, float* out) {
  if (k <= 8 && d <= 128) {
    // On the tensor cores: squared distances |x_i|^2 + |x_j|^2 - 2 x_i.x_j from the tile engine's split-fp16
    // distance GEMM (22 significant bits per coordinate), each row's 8 smallest per column quarter kept in
    // registers (RBF_MODE_KNN), then the quarters merged.  The reference points are gathered and packed as the
    // second point set; their indices skip each point's own distance.
    const int dp = feature_pad(d), npad = point_pad(n), spad = point_pad(s);
    const size_t bytes = 4096 + (size_t)s * d * 4 + (size_t)npad * 2 * dp * 2 + packed_norm_floats(npad) * 4 +
                         (size_t)spad * 2 * dp * 2 + packed_norm_floats(spad) * 4 + (size_t)n * 32 * 4 + 8 * 256;
    char* ws = static_cast<char*>(workspace(ctx, bytes));
    if (!ws) return DB200_ERR_NOMEM;
    Carve cv{ws};
    float* R = cv.take<float>((size_t)s * d);
    void* xq = cv.take<uint16_t>((size_t)npad * 2 * dp);
    float* nq = cv.take<float>(packed_norm_floats(npad));
    void* xr = cv.take<uint16_t>((size_t)spad * 2 * dp);
    float* nr = cv.take<float>(packed_norm_floats(spad));
    float* part = cv.take<float>((size_t)n * 32);
    gather_rows_kernel<<<blocks_for((long long)s * d, 256, 65535LL * 8), 256, 0, ctx->stream>>>(X, ldx, ref, s, d, R);
    DB200_CUDA(ctx, cudaGetLastError());
    count_launch(ctx);
    int st = pack_points(ctx, X, ldx, DB200_POINT_MAJOR, n, d, dp, npad, xq, nq);
    if (!st) st = pack_points(ctx, R, d, DB200_POINT_MAJOR, s, d, dp, spad, xr, nr);
    if (st) return st;
    TileJob J;
    J.pi.xp = xq;
    J.pi.norms = nq;
    J.pi.n = n;
    J.pi.npad = npad;
    J.pi.dp = dp;
    J.pj.xp = xr;
    J.pj.norms = nr;
    J.pj.n = s;
    J.pj.npad = spad;
    J.pj.dp = dp;
    J.yj = reinterpret_cast<const float*>(ref);  // the reference points' indices (RBF_MODE_KNN)
    J.gamma = 1.0f;
    J.out = part;
    J.ldo = 32;
    TilePlan T;
    if ((st = prepare_rbf_tiles(ctx, RBF_MODE_KNN, &J, 1, nullptr, 0, &T))) return st;
    if ((st = launch_rbf_plan(ctx, T))) return st;
    knn_merge_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(n, part, k, out);
    DB200_CUDA(ctx, cudaGetLastError());
    count_launch(ctx);
    return DB200_OK;
  }
  // k > 8: one thread per query on the FP32 pipes
  const unsigned grid = (unsigned)((n + KNN_THREADS - 1) / KNN_THREADS);
  if (d <= 32)
    knn_kernel<32><<<grid, KNN_THREADS, 0, ctx->stream>>>(n, d, X, ldx, s, ref, k, out);
  else if (d <= 64)
    knn_kernel<64><<<grid, KNN_THREADS, 0, ctx->stream>>>(n, d, X, ldx, s, ref, k, out);
  else
    knn_kernel<128><<<grid, KNN_THREADS, 0, ctx->stream>>>(n, d, X, ldx, s, ref, k, out);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

}  // namespace db200

using namespace db200;

extern "C" {

int db200_knn_distance(db200_context* ctx, int n, int d, const float* X, int ldx, int s, const int* ref_idx, int k,
                       float* out) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 0 || d < 1 || d > 128 || ldx < d || s < 1 || k < 1 || k > KNN_KMAX || k > s || !X || !ref_idx || !out)
    return fail(ctx, DB200_ERR_INVALID, "knn_distance: bad arguments (d <= 128, 1 <= k <= min(16, s))");
  if (n == 0) return DB200_OK;
  return knn_distance(ctx, n, d, X, ldx, s, ref_idx, k, out);
}

int db200_leverage_features(db200_context* ctx, int n, int d, const float* X, int ldx, const float* knn, float* F) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 0 || d < 1 || ldx < d || !X || !knn || !F) return fail(ctx, DB200_ERR_INVALID, "leverage_features: bad arguments");
  if (n == 0) return DB200_OK;
  features_kernel<<<blocks_for((long long)n * 32, 256, 65535LL * 8), 256, 0, ctx->stream>>>(n, d, X, ldx, knn, F);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int db200_ridge_leverage(db200_context* ctx, int n, int r, const double* Z, int ldz, double lambda, double* lev) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 1 || r < 1 || ldz < n || !Z || !lev || !(lambda > 0)) return fail(ctx, DB200_ERR_INVALID, "ridge_leverage: bad arguments");
  const size_t rr = (size_t)r * r;
  const size_t bytes = 1024 + 2 * align_up(rr * 8, 256) + align_up((size_t)n * r * 8, 256);
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_SPARE, bytes));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  int* d_pair = cv.take<int>(4);
  double* G = cv.take<double>(rr);
  double* Xi = cv.take<double>(rr);
  double* W = cv.take<double>((size_t)n * r);
  // (Z^T Z + lambda I) = R^T R;  lev_i = ||z_i^T R^-1||^2
  int st = gram<double, double>(ctx, n, r, r, Z, ldz, Z, ldz, nullptr, 1.0, 0.0, G, r, true);
  if (!st) st = mirror_upper(ctx, G, r, r);
  if (!st) st = symmetrize(ctx, G, r, r, lambda);
  if (st) return st;
  DB200_CUDA(ctx, cudaMemsetAsync(d_pair, 0, 2 * sizeof(int), ctx->stream));
  if ((st = potrf_upper(ctx, G, r, r, d_pair, d_pair + 1))) return st;
  int hs[2] = {0, 0};
  DB200_CUDA(ctx, cudaMemcpyAsync(hs, d_pair, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (hs[0]) return fail(ctx, DB200_ERR_NOT_SPD, "ridge_leverage: Z^T Z + lambda I not positive definite");
  if ((st = trinv_upper(ctx, G, r, r, Xi, r))) return st;
  if ((st = gemm_tall<double, double>(ctx, n, r, r, Z, ldz, Xi, r, false, 0.0, W, n))) return st;
  row_sumsq64_kernel<<<blocks_for(n, 256, 4096), 256, 0, ctx->stream>>>(n, r, W, n, lev);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return db200_synchronize(ctx);
}

// ------------------------------------------------------------------ MLP C ABI
int db200_mlp_create(db200_context* ctx, int in_dim, int width, int hidden, unsigned long long seed, db200_mlp** out) {
  if (!ctx || !out) return DB200_ERR_INVALID;
  *out = nullptr;
  if (in_dim < 1 || width < 1 || hidden < 1 || hidden > 7 || in_dim > 4096 || width > 4096)
    return fail(ctx, DB200_ERR_INVALID, "mlp_create: 1 <= hidden <= 7, dims <= 4096");
  db200_mlp* net = new db200_mlp();
  net->in = in_dim;
  net->width = width;
  net->hidden = hidden;
  net->layers = hidden + 1;
  net->device = ctx->device;
  int off = 0;
  for (int l = 0; l < net->layers; ++l) {
    const int fi = (l == 0) ? in_dim : width, fo = (l == hidden) ? 1 : width;
    net->fan_in.push_back(fi);
    net->fan_out.push_back(fo);
    net->off_w.push_back(off);
    off += fi * fo;
    net->off_b.push_back(off);
    off += fo;
  }
  net->nparams = off;
  // He-uniform weights, zero biases (host RNG, seeded)
  std::vector<float> w(off, 0.f);
  std::mt19937_64 g(seed);
  for (int l = 0; l < net->layers; ++l) {
    const float lim = std::sqrt(6.0f / (float)net->fan_in[l]) * (l == hidden ? 0.5f : 1.0f);
    std::uniform_real_distribution<float> u(-lim, lim);
    for (int e = 0; e < net->fan_in[l] * net->fan_out[l]; ++e) w[net->off_w[l] + e] = u(g);
  }
  std::vector<float> mean(in_dim, 0.f), scale(in_dim, 1.f);
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void** p, size_t b) {
    if (e == cudaSuccess) e = cudaMalloc(p, b);
  };
  alloc((void**)&net->master, sizeof(float) * off);
  alloc((void**)&net->grad, sizeof(float) * off);
  alloc((void**)&net->mom1, sizeof(float) * off);
  alloc((void**)&net->mom2, sizeof(float) * off);
  alloc((void**)&net->wbf, sizeof(__nv_bfloat16) * off);
  alloc((void**)&net->in_mean, sizeof(float) * in_dim);
  alloc((void**)&net->in_scale, sizeof(float) * in_dim);
  alloc((void**)&net->d_loss, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(net->master, w.data(), sizeof(float) * off, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(net->mom1, 0, sizeof(float) * off);
  if (e == cudaSuccess) e = cudaMemset(net->mom2, 0, sizeof(float) * off);
  if (e == cudaSuccess) e = cudaMemcpy(net->in_mean, mean.data(), sizeof(float) * in_dim, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(net->in_scale, scale.data(), sizeof(float) * in_dim, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    db200_mlp_destroy(net);
    return cuda_fail(ctx, e, "mlp_create");
  }
  to_bf16_kernel<<<blocks_for(off, 256, 4096), 256, 0, ctx->stream>>>(off, net->master, net->wbf);
  count_launch(ctx);
  DB200_CUDA(ctx, cudaGetLastError());
  *out = net;
  return db200_synchronize(ctx);
}

void db200_mlp_destroy(db200_mlp* net) {
  if (!net) return;
  cudaSetDevice(net->device);
  cudaDeviceSynchronize();
  for (void* p : {(void*)net->master, (void*)net->grad, (void*)net->mom1, (void*)net->mom2, (void*)net->wbf,
                  (void*)net->in_mean, (void*)net->in_scale, (void*)net->d_loss, net->act})
    if (p) cudaFree(p);
  delete net;
}

int db200_mlp_param_count(const db200_mlp* net) { return net ? net->nparams : 0; }

int db200_mlp_get_params(db200_context* ctx, const db200_mlp* net, float* host) {
  if (!ctx || !net || !host) return DB200_ERR_INVALID;
  DB200_CUDA(ctx, cudaMemcpyAsync(host, net->master, sizeof(float) * net->nparams, cudaMemcpyDeviceToHost, ctx->stream));
  return db200_synchronize(ctx);
}

int db200_mlp_set_params(db200_context* ctx, db200_mlp* net, const float* host) {
  if (!ctx || !net || !host) return DB200_ERR_INVALID;
  DB200_CUDA(ctx, cudaMemcpyAsync(net->master, host, sizeof(float) * net->nparams, cudaMemcpyHostToDevice, ctx->stream));
  DB200_CUDA(ctx, cudaMemsetAsync(net->mom1, 0, sizeof(float) * net->nparams, ctx->stream));
  DB200_CUDA(ctx, cudaMemsetAsync(net->mom2, 0, sizeof(float) * net->nparams, ctx->stream));
  net->step = 0;
  to_bf16_kernel<<<blocks_for(net->nparams, 256, 4096), 256, 0, ctx->stream>>>(net->nparams, net->master, net->wbf);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return db200_synchronize(ctx);
}

int db200_mlp_set_input_scaling(db200_context* ctx, db200_mlp* net, const float* mean, const float* scale) {
  if (!ctx || !net || !mean || !scale) return DB200_ERR_INVALID;
  DB200_CUDA(ctx, cudaMemcpyAsync(net->in_mean, mean, sizeof(float) * net->in, cudaMemcpyHostToDevice, ctx->stream));
  DB200_CUDA(ctx, cudaMemcpyAsync(net->in_scale, scale, sizeof(float) * net->in, cudaMemcpyHostToDevice, ctx->stream));
  return db200_synchronize(ctx);
}

int db200_mlp_forward(db200_context* ctx, const db200_mlp* cnet, int m, const float* F, float* out) {
  if (!ctx || !cnet) return DB200_ERR_INVALID;
  if (m < 0 || !F || !out) return fail(ctx, DB200_ERR_INVALID, "mlp_forward: bad arguments");
  if (m == 0) return DB200_OK;
  db200_mlp* net = const_cast<db200_mlp*>(cnet);  // only the grow-only activation buffer changes
  // large m: in chunks so the activations stay bounded
  const int chunk = 1 << 18;
  for (int r0 = 0; r0 < m; r0 += chunk) {
    const int mb = std::min(chunk, m - r0);
    MlpActs A;
    int st = mlp_acts(ctx, net, mb, &A);
    if (!st) st = mlp_forward_impl(ctx, net, mb, F + (size_t)r0 * net->in, A);
    if (st) return st;
    DB200_CUDA(ctx, cudaMemcpyAsync(out + r0, A.out, sizeof(float) * mb, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  return DB200_OK;
}

int db200_mlp_gradients(db200_context* ctx, db200_mlp* net, int m, const float* F, const float* target, float* loss,
                        float* grads) {
  if (!ctx || !net) return DB200_ERR_INVALID;
  if (m < 1 || !F || !target) return fail(ctx, DB200_ERR_INVALID, "mlp_gradients: bad arguments");
  MlpActs A;
  int st = mlp_acts(ctx, net, m, &A);
  if (!st) st = mlp_forward_impl(ctx, net, m, F, A);
  if (!st) st = mlp_backward_impl(ctx, net, m, target, A);
  if (st) return st;
  if (grads)
    DB200_CUDA(ctx, cudaMemcpyAsync(grads, net->grad, sizeof(float) * net->nparams, cudaMemcpyDeviceToDevice, ctx->stream));
  double l = 0;
  DB200_CUDA(ctx, cudaMemcpyAsync(&l, net->d_loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  st = db200_synchronize(ctx);
  if (loss) *loss = (float)l;
  return st;
}

int db200_mlp_adam_step(db200_context* ctx, db200_mlp* net, int m, const float* F, const float* target, float lr,
                        float* loss) {
  if (!ctx || !net) return DB200_ERR_INVALID;
  if (m < 1 || !F || !target || !(lr > 0)) return fail(ctx, DB200_ERR_INVALID, "mlp_adam_step: bad arguments");
  MlpActs A;
  int st = mlp_acts(ctx, net, m, &A);
  if (!st) st = mlp_forward_impl(ctx, net, m, F, A);
  if (!st) st = mlp_backward_impl(ctx, net, m, target, A);
  if (st) return st;
  net->step += 1;
  const float c1 = (float)(1.0 / (1.0 - std::pow(0.9, (double)net->step)));
  const float c2 = (float)(1.0 / (1.0 - std::pow(0.999, (double)net->step)));
  adam_kernel<<<blocks_for(net->nparams, 256, 4096), 256, 0, ctx->stream>>>(net->nparams, net->master, net->grad,
                                                                            net->mom1, net->mom2, net->wbf, lr, c1, c2);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  if (loss) {
    double l = 0;
    DB200_CUDA(ctx, cudaMemcpyAsync(&l, net->d_loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    st = db200_synchronize(ctx);
    *loss = (float)l;
    return st;
  }
  return DB200_OK;
}

// ------------------------------------------------------------------ selection
int db200_gumbel_keys(db200_context* ctx, int n, const float* logits, unsigned long long seed, float* keys) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 0 || !logits || !keys) return fail(ctx, DB200_ERR_INVALID, "gumbel_keys: bad arguments");
  if (n == 0) return DB200_OK;
  gumbel_kernel<<<blocks_for(n, 256, 8192), 256, 0, ctx->stream>>>(n, logits, seed, keys);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int db200_select_topk(db200_context* ctx, int n, const float* keys, int k, int* idx) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 1 || k < 1 || k > n || !keys || !idx) return fail(ctx, DB200_ERR_INVALID, "select_topk: bad arguments");
  unsigned int* buf = static_cast<unsigned int*>(io_buffer(ctx, 4096));
  if (!buf) return DB200_ERR_NOMEM;
  unsigned int prefix = 0, mask = 0;
  int need = k;  // how many still to take at or below the current prefix
  std::vector<unsigned int> h(256);
  const unsigned grid = blocks_for(n, 256, 1024);
  for (int shift = 24; shift >= 0; shift -= 8) {
    DB200_CUDA(ctx, cudaMemsetAsync(buf, 0, 256 * sizeof(unsigned int), ctx->stream));
    radix_hist_kernel<<<grid, 256, 0, ctx->stream>>>(n, keys, prefix, mask, shift, buf);
    DB200_CUDA(ctx, cudaGetLastError());
    count_launch(ctx);
    DB200_CUDA(ctx, cudaMemcpyAsync(h.data(), buf, 256 * sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
    DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    // walk buckets from the top until `need` is covered
    int b = 255;
    for (; b > 0; --b) {
      if ((int)h[b] >= need) break;
      need -= (int)h[b];
    }
    prefix |= (unsigned int)b << shift;
    mask |= 0xFFu << shift;
  }
  // prefix is the k-th largest key; take every key above it and `need` of the keys equal to it
  DB200_CUDA(ctx, cudaMemsetAsync(buf, 0, 2 * sizeof(unsigned int), ctx->stream));
  radix_compact_kernel<<<grid, 256, 0, ctx->stream>>>(n, keys, prefix, need, buf, idx);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  // sorted indices make the landmark order (and so the factor) independent of atomic arrival order
  std::vector<int> hi(k);
  DB200_CUDA(ctx, cudaMemcpyAsync(hi.data(), idx, sizeof(int) * k, cudaMemcpyDeviceToHost, ctx->stream));
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::sort(hi.begin(), hi.end());
  DB200_CUDA(ctx, cudaMemcpyAsync(idx, hi.data(), sizeof(int) * k, cudaMemcpyHostToDevice, ctx->stream));
  return db200_synchronize(ctx);
}

// ------------------------------------------------------------------ landmark factor and residual
}  // extern "C"

// Nystrom factor on landmarks idx; TC = float: C from the tcgen05 tile engine (KBLOCK mode, fp32), TC = double: C
// from the FP64 kernel block (FP64 tensor-core Gram, FP64 exp), the comparator.
template <typename TC>
static int landmark_factor_impl(db200_context* ctx, int n, int d, const float* X, int ldx, const float* y,
                                float gamma, int r, const int* idx, double* Z, int ldz, double* nu_out) {
  const size_t rr = (size_t)r * r;
  const size_t bytes = 4096 + align_up((size_t)n * r * sizeof(TC), 256) + 3 * align_up(rr * 8, 256) +
                       align_up((size_t)r * d * 4, 256) + align_up((size_t)r * 4, 256);
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_PIPE, bytes));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  int* d_pair = cv.take<int>(4);
  double* d_scalar = cv.take<double>(4);
  TC* Cm = cv.take<TC>((size_t)n * r);
  double* W = cv.take<double>(rr);
  double* R = cv.take<double>(rr);
  double* Xinv = cv.take<double>(rr);
  float* XL = cv.take<float>((size_t)r * d);
  float* yL = cv.take<float>(r);
  gather_rows_f32_kernel<<<blocks_for((long long)r * d, 256, 4096), 256, 0, ctx->stream>>>(X, ldx, idx, r, d, XL);
  gather_f32_kernel<<<blocks_for(r, 256, 1024), 256, 0, ctx->stream>>>(y, idx, r, yL);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx, 2);
  // C = diag(y) K(:, L) diag(y_L)
  int st;
  if constexpr (sizeof(TC) == 4)
    st = db200_rbf_block(ctx, n, r, d, X, ldx, XL, d, DB200_POINT_MAJOR, y, yL, Cm, n, gamma);
  else
    st = db200_rbf_block_f64(ctx, n, r, d, X, ldx, XL, d, y, yL, Cm, n, (double)gamma);
  if (st) return st;
  gather_matrix_rows_kernel<TC><<<blocks_for((long long)rr, 256, 4096), 256, 0, ctx->stream>>>(Cm, n, idx, r, r, W);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  if ((st = symmetrize(ctx, W, r, r, 0.0))) return st;
  if ((st = trace(ctx, W, r, r, d_scalar))) return st;
  double tr = 0;
  DB200_CUDA(ctx, cudaMemcpyAsync(&tr, d_scalar, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  double nu = 1e-7 * std::max(tr, 1e-300) / r;
  bool ok = false;
  for (int tries = 0; tries < 12 && !ok; ++tries) {
    DB200_CUDA(ctx, cudaMemcpyAsync(R, W, sizeof(double) * rr, cudaMemcpyDeviceToDevice, ctx->stream));
    if ((st = symmetrize(ctx, R, r, r, nu))) return st;
    DB200_CUDA(ctx, cudaMemsetAsync(d_pair, 0, 2 * sizeof(int), ctx->stream));
    if ((st = potrf_upper(ctx, R, r, r, d_pair, d_pair + 1))) return st;
    int hs[2] = {0, 0};
    DB200_CUDA(ctx, cudaMemcpyAsync(hs, d_pair, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (hs[0] == 0) ok = true;
    else nu *= 10.0;
  }
  if (!ok) return fail(ctx, DB200_ERR_NOT_SPD, "landmark_factor: K(L, L) + nu I not positive definite after 12 shifts");
  // Z = C R^-1
  if ((st = trinv_upper(ctx, R, r, r, Xinv, r))) return st;
  if ((st = gemm_tall<TC, double>(ctx, n, r, r, Cm, n, Xinv, r, false, 0.0, Z, ldz))) return st;
  if (nu_out) *nu_out = nu;
  return db200_synchronize(ctx);
}

extern "C" {

int db200_landmark_factor(db200_context* ctx, int n, int d, const float* X, int ldx, const float* y, float gamma, int r,
                          const int* idx, double* Z, int ldz, double* nu_out) {
  return db200_landmark_factor_ex(ctx, n, d, X, ldx, y, gamma, r, idx, Z, ldz, nu_out, DB200_MIXED);
}

int db200_landmark_factor_ex(db200_context* ctx, int n, int d, const float* X, int ldx, const float* y, float gamma,
                             int r, const int* idx, double* Z, int ldz, double* nu_out, int precision) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 1 || d < 1 || d > 128 || ldx < d || r < 1 || r > n || !X || !y || !idx || !Z || ldz < n ||
      (precision != DB200_MIXED && precision != DB200_FP64 && precision != DB200_MIXED_FAST))
    return fail(ctx, DB200_ERR_INVALID, "landmark_factor: bad arguments");
  return precision == DB200_FP64 ? landmark_factor_impl<double>(ctx, n, d, X, ldx, y, gamma, r, idx, Z, ldz, nu_out)
                                 : landmark_factor_impl<float>(ctx, n, d, X, ldx, y, gamma, r, idx, Z, ldz, nu_out);
}

int db200_residual_estimate(db200_context* ctx, int n, int d, const float* X, int ldx, const float* y, float gamma,
                            int r, const double* Z, int ldz, int s, const int* sample_idx, double* est) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 1 || d < 1 || d > 128 || ldx < d || r < 1 || s < 1 || s > n || !X || !y || !Z || ldz < n || !sample_idx ||
      !est)
    return fail(ctx, DB200_ERR_INVALID, "residual_estimate: bad arguments");
  const size_t bytes = 4096 + align_up((size_t)n * s * 4, 256) + align_up((size_t)n * s * 8, 256) +
                       align_up((size_t)s * r * 8, 256) + align_up((size_t)s * d * 4, 256) + align_up((size_t)s * 4, 256);
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_SPARE, bytes));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  double* sums = cv.take<double>(4);
  float* Ks = cv.take<float>((size_t)n * s);
  double* T = cv.take<double>((size_t)n * s);
  double* Zs = cv.take<double>((size_t)s * r);
  float* Xs = cv.take<float>((size_t)s * d);
  float* ys = cv.take<float>(s);
  gather_rows_f32_kernel<<<blocks_for((long long)s * d, 256, 4096), 256, 0, ctx->stream>>>(X, ldx, sample_idx, s, d, Xs);
  gather_f32_kernel<<<blocks_for(s, 256, 1024), 256, 0, ctx->stream>>>(y, sample_idx, s, ys);
  gather_matrix_rows_kernel<double><<<blocks_for((long long)s * r, 256, 4096), 256, 0, ctx->stream>>>(Z, ldz, sample_idx,
                                                                                                     s, r, Zs);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx, 3);
  int st = db200_rbf_block(ctx, n, s, d, X, ldx, Xs, d, DB200_POINT_MAJOR, y, ys, Ks, n, gamma);
  if (st) return st;
  // T = Z Z(S, :)^T (n x s)
  if ((st = gemm_tall<double, double>(ctx, n, r, s, Z, ldz, Zs, s, true, 0.0, T, n))) return st;
  DB200_CUDA(ctx, cudaMemsetAsync(sums, 0, 2 * sizeof(double), ctx->stream));
  if ((st = sumsq_f32(ctx, Ks, n, n, s, sums))) return st;
  if ((st = axpby_f32(ctx, Ks, n, T, n, n, s, -1.0, 1.0))) return st;
  if ((st = sumsq_f32(ctx, Ks, n, n, s, sums + 1))) return st;
  double hs[2] = {0, 0};
  DB200_CUDA(ctx, cudaMemcpyAsync(hs, sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  st = db200_synchronize(ctx);
  if (st) return st;
  *est = (hs[0] > 0) ? std::sqrt(hs[1] / hs[0]) : 0.0;
  return DB200_OK;
}

// ------------------------------------------------------------------ the learned-landmark solve
// Landmark selection of the learned solve: k-NN features over sk reference points -> MLP log-leverage -> Gumbel
// keys -> top r.  Scratch F, knn, logits, keys, ref come from the caller's carve; idx receives r device indices.
static int select_landmarks_impl(db200_context* ctx, int n, int d, int r, const float* X, int ldx, const db200_mlp* net,
                                 unsigned long long seed, int sk, float* F, float* knn, float* logits, float* keys,
                                 int* ref, int* idx, db200_landmark_report* L) {
  const std::vector<int> h_ref = sample_indices(n, sk, seed ^ 0x6b6e6eull);
  DB200_CUDA(ctx, cudaMemcpyAsync(ref, h_ref.data(), sizeof(int) * sk, cudaMemcpyHostToDevice, ctx->stream));
  int st;
  {
    LandTimer t(ctx->stream);
    if ((st = knn_distance(ctx, n, d, X, ldx, sk, ref, 8, knn))) return st;
    if ((st = db200_leverage_features(ctx, n, d, X, ldx, knn, F))) return st;
    L->ms_features = t.stop();
  }
  {
    LandTimer t(ctx->stream);
    if ((st = db200_mlp_forward(ctx, net, n, F, logits))) return st;
    L->ms_predict = t.stop();
  }
  {
    LandTimer t(ctx->stream);
    if ((st = db200_gumbel_keys(ctx, n, logits, seed, keys))) return st;
    if ((st = db200_select_topk(ctx, n, keys, r, idx))) return st;
    L->ms_select = t.stop();
  }
  return DB200_OK;
}

int db200_select_landmarks(db200_context* ctx, int n, int d, int r, const float* X, int ldx, const db200_mlp* net,
                           unsigned long long seed, int s_knn, int* idx) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 2 || d < 1 || d > 128 || ldx < d || r < 1 || r > n || !X || !net || net->in != d + 2 || s_knn < 9 || !idx)
    return fail(ctx, DB200_ERR_INVALID, "select_landmarks: bad arguments (model input must be d + 2)");
  const int sk = std::min(s_knn, n);
  const size_t bytes = 4096 + align_up((size_t)n * (d + 2) * 4, 256) + 3 * align_up((size_t)n * 4, 256) +
                       align_up((size_t)sk * 4, 256);
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_LAND, bytes));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  float* F = cv.take<float>((size_t)n * (d + 2));
  float* knn = cv.take<float>(n);
  float* logits = cv.take<float>(n);
  float* keys = cv.take<float>(n);
  int* ref = cv.take<int>(sk);
  db200_landmark_report L;
  std::memset(&L, 0, sizeof(L));
  int st = select_landmarks_impl(ctx, n, d, r, X, ldx, net, seed, sk, F, knn, logits, keys, ref, idx, &L);
  if (st) return st;
  return db200_synchronize(ctx);
}

int db200_svm_solve_landmarks(db200_context* ctx, int n, int d, int r, const float* X, int ldx, const float* y,
                              float gamma, double C, const db200_mlp* net, unsigned long long seed, int s_knn,
                              int s_res, double tol, const float* Omega, int ldo, int l_fb, int q,
                              const db200_barrier_params* params, double* a, double* Z, int ldz, db200_svm_report* rep,
                              db200_landmark_report* lrep) {
  if (!ctx) return DB200_ERR_INVALID;
  if (sharded(ctx))
    return fail(ctx, DB200_ERR_UNSUPPORTED, "svm_solve_landmarks: not row-sharded (detach the collective first)");
  if (n < 2 || d < 1 || d > 128 || ldx < d || r < 1 || r > n || !X || !y || !net || net->in != d + 2 || s_knn < 9 ||
      s_res < 1 || !a || !Z || ldz < n || (Omega && (ldo < n || l_fb < 1 || l_fb > n)) || q < 0)
    return fail(ctx, DB200_ERR_INVALID, "svm_solve_landmarks: bad arguments (model input must be d + 2)");
  db200_landmark_report L;
  std::memset(&L, 0, sizeof(L));
  db200_svm_report R;
  std::memset(&R, 0, sizeof(R));
  LandTimer total(ctx->stream);
  const int sk = std::min(s_knn, n), sr = std::min(s_res, n);
  const size_t bytes = 4096 + align_up((size_t)n * (d + 2) * 4, 256) + 3 * align_up((size_t)n * 4, 256) +
                       align_up((size_t)r * 4, 256) + align_up((size_t)sk * 4, 256) + align_up((size_t)sr * 4, 256);
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_LAND, bytes));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  float* F = cv.take<float>((size_t)n * (d + 2));
  float* knn = cv.take<float>(n);
  float* logits = cv.take<float>(n);
  float* keys = cv.take<float>(n);
  int* idx = cv.take<int>(r);
  int* ref = cv.take<int>(sk);
  int* res = cv.take<int>(sr);
  const std::vector<int> h_res = sample_indices(n, sr, seed ^ 0x726573ull);
  DB200_CUDA(ctx, cudaMemcpyAsync(res, h_res.data(), sizeof(int) * sr, cudaMemcpyHostToDevice, ctx->stream));
  int st = select_landmarks_impl(ctx, n, d, r, X, ldx, net, seed, sk, F, knn, logits, keys, ref, idx, &L);
  if (st) return st;
  {
    LandTimer t(ctx->stream);
    double nu = 0;
    // The landmark columns C = K(:, L) cost n r d, a fraction r / n of one Gaussian kernel pass: the parity-grade
    // mixed form (and the FP64 one) takes them in FP64, whose factor then matches the FP64 Nystrom factor on the
    // same landmarks to round-off; the fast mixed form takes the tile engine's fp32 block (~1e-6 from FP64 in f).
    db200_barrier_params Pf;
    if (params) Pf = *params;
    else db200_barrier_defaults(&Pf);
    const int cprec = (Pf.precision == DB200_MIXED_FAST) ? DB200_MIXED_FAST : DB200_FP64;
    if ((st = db200_landmark_factor_ex(ctx, n, d, X, ldx, y, gamma, r, idx, Z, ldz, &nu, cprec))) return st;
    R.nu = nu;
    L.ms_factor = t.stop();
  }
  {
    LandTimer t(ctx->stream);
    if ((st = db200_residual_estimate(ctx, n, d, X, ldx, y, gamma, r, Z, ldz, sr, res, &L.residual_est))) return st;
    L.ms_residual = t.stop();
  }
  int rank = r;
  if (!(L.residual_est <= tol) && Omega) {
    // fall back to the Gaussian sketch
    LandTimer t(ctx->stream);
    L.used_fallback = 1;
    db200_barrier_params P;
    if (params) P = *params;
    else db200_barrier_defaults(&P);
    if ((st = db200_lowrank(ctx, n, d, l_fb, q, X, ldx, y, Omega, ldo, gamma, P.precision, Z, ldz, &R))) return st;
    rank = l_fb;
    if ((st = db200_residual_estimate(ctx, n, d, X, ldx, y, gamma, rank, Z, ldz, sr, res, &L.residual_fallback)))
      return st;
    L.ms_fallback = t.stop();
  }
  L.rank = rank;
  const double nu_keep = R.nu;
  st = db200_svm_barrier(ctx, n, rank, Z, ldz, y, C, params, a, &R);
  if (st && st != DB200_ERR_MAXITER) return st;
  if (!L.used_fallback) R.nu = nu_keep;
  R.ms_total = total.stop();
  if (rep) *rep = R;
  if (lrep) *lrep = L;
  return st;
}

}  // extern "C"
