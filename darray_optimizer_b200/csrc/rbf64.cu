// Plain-FP64 fused RBF kernel x sketch, the comparator of the mixed-precision tile engine:
//     Y(m x l) = diag(yi) K(Xi, Xj) diag(yj) Omega,   K(a, b) = exp(-gamma max(s_a + s_b - 2 x_a.x_b, 0))
// with FP64 norms, distances, exp and products; K is never stored.  The same GEMM form as include/dkernel.cu:116-129
// (vecnorm, rbf) and the sketch product of :194-231 / include/dkernel.h:13-46, in FP64 throughout.
//
// One CTA (8 warps) owns 64 rows of i and one tile of up to 264 sketch columns and streams all points j in stages
// of 16 (two K steps of mma.sync.m16n8k8.f64).  Per stage every warp w does the same DMMA work:
//   distance  G(16 x 8) = Xi . Xj^T over d for row tile w % 4 and the 8 points 8 (w / 4).. of the stage (d/8 DMMAs
//             in two chains), then K = exp(-gamma max(s_i + s_j - 2 G, 0)) in FP64 into a shared 64 x 16 tile
//   sketch    Y(16 x LT/2) += K(16 x 16) . Omega~(16 x LT/2): row tile w % 4, column half w / 4 (two K steps)
// so the eight warps issue equal DMMA counts and only one barrier per 16 points is needed.  Xi lives in shared
// memory in FP64 for the whole CTA; Xj (fp32) and Omega~ stages arrive by cp.async into double buffers, Xj two
// stages ahead and Omega~ one: the distance of stage s + 1 is computed while the sketch of stage s runs.
// Omega~ = diag(yj) Omega is pre-blocked [n/16][lpad][16] so each stage is one contiguous block.
//
// Issued work per 64 rows and 16 points: 8 d/8 distance DMMAs + 8 LT/8 sketch DMMAs per sketch tile; at d = 128,
// l = 528 (two tiles of 264) that is 1.2x the algorithmic 2 n^2 (d + l) flops (the distance is recomputed per tile).
#include <cmath>

#include "internal.h"
#include "la64.h"

namespace db200 {
namespace {

constexpr int R64_ROWS = 64;      // rows of i per CTA
constexpr int R64_THREADS = 256;  // 8 warps
constexpr int R64_KS = 16;        // points j per stage
constexpr int R64_KPAD = 20;      // padded row of 16 doubles (K tile, Omega~ stage): conflict-free fragments

__device__ __forceinline__ void dmma(double* d, const double* a, const double* b) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, bool valid) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  const int n = valid ? 4 : 0;  // src-size 0: the destination is zero-filled
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

struct R64Args {
  int m, n, d, dp, l, lpad, lt, n_ltiles, n_stages;
  const float* Xi;
  long long ldxi;
  const float* Xj;
  long long ldxj;
  const double* si;  // FP64 squared norms
  const double* sj;  // padded with zeros to n_stages * 16
  const float* yi;
  const double* Ob;  // [n_stages][lpad][16] = y_j Omega(j, c), zero for j >= n or c >= l
  double gamma;
  double* Y;
  long long ldy;
};

// Shared layout (doubles): Xi [64][dp + 4] | K [2][64][20] | Omega~ [2][lt][20]; Xj (floats) [2][16][dp + 4].
__host__ __device__ inline size_t r64_smem_bytes(int dp, int lt) {
  return 8 * ((size_t)R64_ROWS * (dp + 4) + 2 * R64_ROWS * R64_KPAD + 2 * (size_t)lt * R64_KPAD) +
         4 * 2 * (size_t)R64_KS * (dp + 4);
}

// NT = n8 column tiles of the CTA's sketch tile (LT = 8 NT); warp half 0 holds tiles [0, H0), half 1 [H0, NT).
template <int NT>
__global__ void __launch_bounds__(R64_THREADS, 1) rbf_sketch_f64_kernel(const R64Args a) {
  constexpr int H0 = (NT + 1) / 2, H1 = NT - H0, NB = H0;  // accumulator tiles per warp (half 1 uses H1 <= NB)
  extern __shared__ __align__(16) double smem64[];
  const int dp = a.dp, S = dp + 4, lt = 8 * NT;
  double* sXi = smem64;
  double* sK = sXi + (size_t)R64_ROWS * S;
  double* sO = sK + 2 * R64_ROWS * R64_KPAD;
  float* sXj = reinterpret_cast<float*>(sO + 2 * (size_t)lt * R64_KPAD);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int g = lane / 4, t = lane % 4;
  const int mt = warp & 3, half = warp >> 2;  // row tile (16 rows); column half (sketch) / point half (distance)
  const int nb0 = half ? H0 : 0, nbn = half ? H1 : H0;
  const int i0 = (blockIdx.x / a.n_ltiles) * R64_ROWS;
  const int lt_idx = blockIdx.x % a.n_ltiles;
  const int c0 = lt_idx * lt;  // first sketch column of this tile (Ob rows)

  // Xi rows in FP64, zero padded (rows >= m, features >= d)
  for (int e = threadIdx.x; e < R64_ROWS * dp; e += R64_THREADS) {
    const int r = e / dp, k = e % dp;
    const int i = i0 + r;
    sXi[r * S + k] = (i < a.m && k < a.d) ? (double)a.Xi[(long long)i * a.ldxi + k] : 0.0;
  }

  // copies of one stage's Xj rows j0..j0+15 (fp32, zero-filled past n and d) into buffer s & 1
  auto issue_xj = [&](int s) {
    const int j0 = s * R64_KS;
    float* dst = sXj + (size_t)(s & 1) * R64_KS * S;
    for (int e = threadIdx.x; e < R64_KS * dp; e += R64_THREADS) {
      const int r = e / dp, k = e % dp;
      const int j = j0 + r;
      const bool ok = j < a.n && k < a.d;
      cp_async4(dst + r * S + k, ok ? (const void*)(a.Xj + (long long)j * a.ldxj + k) : (const void*)a.Xj, ok);
    }
  };
  // copies of one stage's Omega~ block of this tile into buffer s & 1: 8 pieces of 16 bytes per column
  auto issue_om = [&](int s) {
    const double* src = a.Ob + ((size_t)s * a.lpad + c0) * R64_KS;
    double* od = sO + (size_t)(s & 1) * lt * R64_KPAD;
    for (int e = threadIdx.x; e < lt * 8; e += R64_THREADS) {
      const int c = e >> 3, q = e & 7;
      cp_async16(od + c * R64_KPAD + 2 * q, src + (size_t)c * R64_KS + 2 * q);
    }
  };

  // distance of stage s for row tile mt and points 8 half.. of the stage, exp, into K buffer s & 1
  const int rA = 16 * mt + g;  // this lane's fragment rows rA, rA + 8
  const double si0 = (i0 + rA < a.m) ? a.si[i0 + rA] : 0.0;
  const double si1 = (i0 + rA + 8 < a.m) ? a.si[i0 + rA + 8] : 0.0;
  auto distance = [&](int s) {
    const float* xj = sXj + (size_t)(s & 1) * R64_KS * S + (size_t)(8 * half) * S;
    double c[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};  // two independent chains over k
    for (int k0 = 0; k0 < dp; k0 += 16) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int k = k0 + 8 * h;
        if (k < dp) {
          double af[4], bf[2];
          af[0] = sXi[rA * S + k + t];
          af[1] = sXi[(rA + 8) * S + k + t];
          af[2] = sXi[rA * S + k + t + 4];
          af[3] = sXi[(rA + 8) * S + k + t + 4];
          bf[0] = (double)xj[g * S + k + t];
          bf[1] = (double)xj[g * S + k + t + 4];
          dmma(c[h], af, bf);
        }
      }
    }
    // c[.][0,1] = G(rA, 2t + 0/1), c[.][2,3] = G(rA + 8, 2t + 0/1) for the points 8 half + 2t + 0/1
    const int jl = 8 * half + 2 * t;  // column inside the stage's K tile
    const int j0 = s * R64_KS + jl;
    const double sj0 = a.sj[j0], sj1 = a.sj[j0 + 1];
    double* kt = sK + (size_t)(s & 1) * R64_ROWS * R64_KPAD;
    const double G00 = c[0][0] + c[1][0], G01 = c[0][1] + c[1][1];
    const double G10 = c[0][2] + c[1][2], G11 = c[0][3] + c[1][3];
    kt[rA * R64_KPAD + jl] = exp(-a.gamma * fmax(si0 + sj0 - 2.0 * G00, 0.0));
    kt[rA * R64_KPAD + jl + 1] = exp(-a.gamma * fmax(si0 + sj1 - 2.0 * G01, 0.0));
    kt[(rA + 8) * R64_KPAD + jl] = exp(-a.gamma * fmax(si1 + sj0 - 2.0 * G10, 0.0));
    kt[(rA + 8) * R64_KPAD + jl + 1] = exp(-a.gamma * fmax(si1 + sj1 - 2.0 * G11, 0.0));
  };

  double acc[NB][4];
#pragma unroll
  for (int b = 0; b < NB; ++b)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[b][e] = 0.0;

  const int S_n = a.n_stages;
  issue_xj(0);
  if (S_n > 1) issue_xj(1);
  issue_om(0);
  cp_async_commit();
  cp_async_wait_all();
  __syncthreads();  // Xi, Xj(0), Xj(1), Omega~(0)
  distance(0);
  for (int s = 0; s < S_n; ++s) {
    cp_async_wait_all();  // this thread's copies of Xj(s + 1) and Omega~(s) (issued one iteration ago)
    __syncthreads();      // K(s) complete and every copy visible; every read of stage s - 1 done
    // Xj(s + 2) reuses the buffer distance(s) read (iteration s - 1); Omega~(s + 1) the one sketch(s - 1) read
    if (s + 2 < S_n) issue_xj(s + 2);
    if (s + 1 < S_n) issue_om(s + 1);
    cp_async_commit();
    // sketch of stage s: two K steps of 8 points
    {
      const double* kt = sK + (size_t)(s & 1) * R64_ROWS * R64_KPAD;
      const double* ot = sO + (size_t)(s & 1) * lt * R64_KPAD;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        double af[4];
        af[0] = kt[rA * R64_KPAD + 8 * ks + t];
        af[1] = kt[(rA + 8) * R64_KPAD + 8 * ks + t];
        af[2] = kt[rA * R64_KPAD + 8 * ks + t + 4];
        af[3] = kt[(rA + 8) * R64_KPAD + 8 * ks + t + 4];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          if (half == 0 || b < H1) {  // uniform per warp; half 1 holds H1 = NB or NB - 1 tiles
            const int col = 8 * (nb0 + b) + g;
            double bf[2] = {ot[col * R64_KPAD + 8 * ks + t], ot[col * R64_KPAD + 8 * ks + t + 4]};
            dmma(acc[b], af, bf);
          }
        }
      }
    }
    if (s + 1 < S_n) distance(s + 1);
  }
  cp_async_wait_all();

  // Y(i, c) = y_i acc
  const int ia = i0 + rA, ib = ia + 8;
  const double ya = (ia < a.m) ? (a.yi ? (double)a.yi[ia] : 1.0) : 0.0;
  const double yb = (ib < a.m) ? (a.yi ? (double)a.yi[ib] : 1.0) : 0.0;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    if (b >= nbn) continue;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int c = c0 + 8 * (nb0 + b) + 2 * t + e;
      if (c >= a.l) continue;
      if (ia < a.m) a.Y[(long long)c * a.ldy + ia] = ya * acc[b][e];
      if (ib < a.m) a.Y[(long long)c * a.ldy + ib] = yb * acc[b][2 + e];
    }
  }
}

// Ob[s][c][jj] = y_j Omega(j, c) for j = 16 s + jj < n and c < l, else 0
__global__ void block_omega_kernel(const double* __restrict__ Om, long long ldo, const float* __restrict__ yj, int n,
                                   int l, int lpad, int n_stages, double* __restrict__ Ob) {
  const long long total = (long long)n_stages * lpad * R64_KS;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int jj = (int)(e % R64_KS);
    const long long sc = e / R64_KS;
    const int c = (int)(sc % lpad);
    const int s = (int)(sc / lpad);
    const int j = R64_KS * s + jj;
    double v = 0.0;
    if (j < n && c < l) v = Om[(long long)c * ldo + j] * (yj ? (double)yj[j] : 1.0);
    Ob[e] = v;
  }
}

template <int NT>
cudaError_t launch_r64(const R64Args& a, int blocks, size_t smem, cudaStream_t st) {
  auto k = rbf_sketch_f64_kernel<NT>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<blocks, R64_THREADS, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace

// Sketch tile width: up to 264 columns (33 n8 tiles) per CTA; small sketches, and wide points whose Xi tile
// leaves too little shared memory, take narrower tiles.
constexpr size_t R64_SMEM_MAX = 227 * 1024;
static int r64_tile_cols(int l, int dp) {
  if (l <= 16 || r64_smem_bytes(dp, 144) > R64_SMEM_MAX) return 16;
  if (l <= 144 || r64_smem_bytes(dp, 264) > R64_SMEM_MAX) return 144;
  return 264;
}

int rbf_sketch_f64_fused(db200_context* ctx, int m, int n, int d, int l, const float* Xi, int ldxi, const float* Xj,
                         int ldxj, const float* yi, const float* yj, const double* Omega, int ldo, double* Y, int ldy,
                         double gamma) {
  const int dp = round_up(d, 8);
  const int lt = r64_tile_cols(l, dp);
  const int n_lt = (l + lt - 1) / lt;
  const int lpad = n_lt * lt;
  const int n_stages = (n + R64_KS - 1) / R64_KS;
  const size_t smem = r64_smem_bytes(dp, lt);
  if (smem > R64_SMEM_MAX) return fail(ctx, DB200_ERR_UNSUPPORTED, "rbf_sketch_f64: d too large for the FP64 tile");
  const size_t bytes = 1024 + align_up((size_t)m * 8, 256) + align_up((size_t)n_stages * R64_KS * 8, 256) +
                       align_up((size_t)n_stages * lpad * R64_KS * 8, 256) + 1024;
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_SPARE, bytes));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  double* si = cv.take<double>(m);
  double* sj = cv.take<double>((size_t)n_stages * R64_KS);
  double* Ob = cv.take<double>((size_t)n_stages * lpad * R64_KS);
  DB200_CUDA(ctx, cudaMemsetAsync(sj, 0, sizeof(double) * (size_t)n_stages * R64_KS, ctx->stream));
  int st = rownorm_f64(ctx, Xi, ldxi, m, d, si);
  if (!st) st = rownorm_f64(ctx, Xj, ldxj, n, d, sj);
  if (st) return st;
  {
    const long long total = (long long)n_stages * lpad * R64_KS;
    long long blocks = (total + 255) / 256;
    if (blocks > (long long)ctx->num_sms * 32) blocks = (long long)ctx->num_sms * 32;
    block_omega_kernel<<<(unsigned)blocks, 256, 0, ctx->stream>>>(Omega, ldo, yj, n, l, lpad, n_stages, Ob);
    DB200_CUDA(ctx, cudaGetLastError());
    count_launch(ctx);
  }
  R64Args a;
  a.m = m;
  a.n = n;
  a.d = d;
  a.dp = dp;
  a.l = l;
  a.lpad = lpad;
  a.lt = lt;
  a.n_ltiles = n_lt;
  a.n_stages = n_stages;
  a.Xi = Xi;
  a.ldxi = ldxi;
  a.Xj = Xj;
  a.ldxj = ldxj;
  a.si = si;
  a.sj = sj;
  a.yi = yi;
  a.Ob = Ob;
  a.gamma = gamma;
  a.Y = Y;
  a.ldy = ldy;
  const int blocks = ((m + R64_ROWS - 1) / R64_ROWS) * n_lt;
  cudaEvent_t e0 = nullptr;
  prof_begin(ctx, &e0);
  cudaError_t e = (lt == 264)   ? launch_r64<33>(a, blocks, smem, ctx->stream)
                  : (lt == 144) ? launch_r64<18>(a, blocks, smem, ctx->stream)
                                : launch_r64<2>(a, blocks, smem, ctx->stream);
  DB200_CUDA(ctx, e);
  prof_end(ctx, e0);
  count_launch(ctx);
  return DB200_OK;
}

}  // namespace db200
