// FP64 dense linear algebra for the 1 x 1 DMatrix path: tall-skinny Gram (matrix_multiply T,N), tall GEMM,
// blocked Cholesky (cholesky_factorize 'U'), triangular inverse / solves (triangular_solve), GEMV pairs.
//
// Restated from include/lapack_like.h:10-56 (blocked right-looking Cholesky: potrf on the diagonal block, trsm on
// the panel, syrk on the trailing matrix), include/blas_like.h:63-127 (matrix_multiply T,N; triangular_solve
// L,U,T,N) and include/cblas_like.h:40-69, in FP64 on the GPU.  All matrices are column major.
#include <cstdio>
#include <type_traits>

#include "internal.h"
#include "la64.h"

namespace db200 {

namespace {

template <typename T>
__device__ __forceinline__ double ld64(const T* p) { return (double)__ldg(p); }

// C[p x q] (+)= alpha * A^T diag(w) B over rows [r0, r1) of A (n x p) and B (n x q); FP64 accumulation.
// grid.z splits the rows; partial tiles are added with FP64 atomics when grid.z > 1.
//
// FP64 tensor cores (mma.sync.m16n8k8.f64): 128 x 128 output tile per CTA, 8 warps of 32 x 64 (2 x 8 MMA tiles,
// 64 accumulators per thread).  Stages of 8 rows of A and B are fetched into registers one stage ahead (coalesced
// column reads: consecutive threads walk consecutive rows) and parked transposed (k-major) in a double-buffered
// shared tile; per stage a warp loads 2 A fragments (4 doubles each) and 8 B fragments (2 doubles each) for 16
// MMAs.  Fragment layouts of m16n8k8 (g = lane / 4, t = lane % 4): A (16 x 8, row) a0..a3 = A[g][t], A[g+8][t],
// A[g][t+4], A[g+8][t+4]; B (8 x 8, col) b0, b1 = B[t][g], B[t+4][g]; C (16 x 8) c0, c1 = C[g][2t + 0, 1],
// c2, c3 = C[g+8][2t + 0, 1].
constexpr int GT = 128;        // Gram output tile
constexpr int GK = 8;          // rows per stage
constexpr int GPAD = GT + 8;   // padded shared row: 4 consecutive k rows land 16 banks apart

__device__ __forceinline__ void dmma16(double* d, const double* a, const double* b) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

constexpr int GTHREADS = 256;

template <typename TA, typename TBt>
__global__ void __launch_bounds__(GTHREADS, 1) gram_kernel(int n, int p, int q, const TA* __restrict__ A, long long lda,
                                                      const TBt* __restrict__ B, long long ldb,
                                                      const double* __restrict__ w, double alpha, double* C, int ldc,
                                                      int rows_per_split, int upper_only, int atomic) {
  const int bi = blockIdx.x, bj = blockIdx.y;
  if (upper_only && bi > bj) return;
  const int i0 = bi * GT, j0 = bj * GT;
  const int r0 = blockIdx.z * rows_per_split;
  const int r1 = min(n, r0 + rows_per_split);
  __shared__ __align__(16) double sA[2][GK][GPAD];
  __shared__ __align__(16) double sB[2][GK][GPAD];
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  const int wm = warp / 2, wn = warp % 2;  // warp tile: rows 32 wm .. +31, columns 64 wn .. +63
  const int fr = lane / 4, fk = lane % 4;  // fragment row / k index of this lane
  double acc[2][8][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[a][b][e] = 0.0;
  const int kk = threadIdx.x % GK;   // row inside the stage this thread loads
  const int c0 = threadIdx.x / GK;   // first column it loads (then +32, +64, +96)
  double va[4], vb[4];
  auto fetch = [&](int k0) {
    const int k = k0 + kk;
    const bool kin = k < r1;
    const double wk = (w && kin) ? w[k] : 1.0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int c = c0 + 32 * s;
      const int ia = i0 + c, jb = j0 + c;
      va[s] = (kin && ia < p) ? wk * ld64(A + (long long)ia * lda + k) : 0.0;
      vb[s] = (kin && jb < q) ? ld64(B + (long long)jb * ldb + k) : 0.0;
    }
  };
  auto park = [&](int buf) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      sA[buf][kk][c0 + 32 * s] = va[s];
      sB[buf][kk][c0 + 32 * s] = vb[s];
    }
  };
  int buf = 0;
  if (r0 < r1) {
    fetch(r0);
    park(0);
  }
  __syncthreads();
  for (int k0 = r0; k0 < r1; k0 += GK) {
    // the next stage's global loads are in flight while this stage is multiplied
    const bool more = k0 + GK < r1;
    if (more) fetch(k0 + GK);
    {
      double af[2][4], bf[8][2];
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        const int r = 32 * wm + 16 * a + fr;
        af[a][0] = sA[buf][fk][r];
        af[a][1] = sA[buf][fk][r + 8];
        af[a][2] = sA[buf][fk + 4][r];
        af[a][3] = sA[buf][fk + 4][r + 8];
      }
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int c = 64 * wn + 8 * b + fr;
        bf[b][0] = sB[buf][fk][c];
        bf[b][1] = sB[buf][fk + 4][c];
      }
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) dmma16(acc[a][b], af[a], bf[b]);
    }
    if (more) park(buf ^ 1);  // the other buffer was last read one stage ago, before the barrier below
    __syncthreads();
    buf ^= 1;
  }
#pragma unroll
  for (int a = 0; a < 2; ++a) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = i0 + 32 * wm + 16 * a + 8 * h + fr;
      if (i >= p) continue;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int j = j0 + 64 * wn + 8 * b + 2 * fk + e;
          if (j >= q) continue;
          if (upper_only && i > j) continue;
          double* dst = C + (long long)j * ldc + i;
          const double v = alpha * acc[a][b][2 * h + e];
          if (atomic)
            atomicAdd(dst, v);
          else
            *dst += v;
        }
      }
    }
  }
}

// The same Gram for FP64 operands with 16-byte-aligned columns (base and leading dimensions), as a cp.async
// pipeline: 16-row stages of A's and B's 128 columns land column-major in shared memory (padded so that the
// fragment loads of a warp spread over the banks), GP_STAGES deep, while the 8 warps run the DMMA tiles of the
// stage before; a stage's rows past the split's end or columns past p / q are zero-filled by the copy.  The weights
// scale A's fragments.  Same tiles, accumulators and epilogue as gram_kernel.
constexpr int GP_KS = 16;                   // rows per stage
constexpr int GP_KPAD = GP_KS + 4;          // doubles per staged column (= 4 mod 16: conflict-free fragment loads)
constexpr int GP_STAGES = 4;
constexpr int GP_STAGE_DOUBLES = 2 * GT * GP_KPAD;  // A and B
constexpr size_t GP_SMEM = (size_t)GP_STAGES * GP_STAGE_DOUBLES * sizeof(double);

__device__ __forceinline__ void gp_cp16(double* smem, const double* gmem, int valid_doubles) {
  const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  const int bytes = valid_doubles <= 0 ? 0 : (valid_doubles >= 2 ? 16 : 8);  // the rest zero-filled
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sa), "l"(gmem), "r"(bytes) : "memory");
}

__global__ void __launch_bounds__(GTHREADS, 1) gram_pipe_kernel(int n, int p, int q, const double* __restrict__ A,
                                                               long long lda, const double* __restrict__ B,
                                                               long long ldb, const double* __restrict__ w,
                                                               double alpha, double* C, int ldc, int rows_per_split,
                                                               int upper_only, int atomic) {
  const int bi = blockIdx.x, bj = blockIdx.y;
  if (upper_only && bi > bj) return;
  extern __shared__ __align__(16) double gsm[];
  const int i0 = bi * GT, j0 = bj * GT;
  const int r0 = blockIdx.z * rows_per_split;
  const int r1 = min(n, r0 + rows_per_split);
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  const int wm = warp / 2, wn = warp % 2;  // warp tile: rows 32 wm .. +31, columns 64 wn .. +63
  const int fr = lane / 4, fk = lane % 4;
  const int nst = (r1 > r0) ? (r1 - r0 + GP_KS - 1) / GP_KS : 0;
  // stage s: rows r0 + 16 s .. + 15; each thread copies 4 chunks of A and 4 of B (16 B = 2 rows of one column)
  auto issue = [&](int st) {
    double* sA = gsm + (size_t)(st % GP_STAGES) * GP_STAGE_DOUBLES;
    double* sB = sA + GT * GP_KPAD;
    const int kbase = r0 + st * GP_KS;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = threadIdx.x + GTHREADS * u;  // 0 .. 1023: column e / 8, row pair e % 8
      const int c = e >> 3, kp = (e & 7) * 2;
      const int k = kbase + kp;
      const int valid = (k < r1) ? min(2, r1 - k) : 0;
      const int ia = i0 + c, jb = j0 + c;
      gp_cp16(sA + c * GP_KPAD + kp, (ia < p && valid) ? A + (long long)ia * lda + k : A, ia < p ? valid : 0);
      gp_cp16(sB + c * GP_KPAD + kp, (jb < q && valid) ? B + (long long)jb * ldb + k : B, jb < q ? valid : 0);
    }
  };
  double acc[2][8][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[a][b][e] = 0.0;
#pragma unroll
  for (int st = 0; st < GP_STAGES - 1; ++st) {
    if (st < nst) issue(st);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  for (int st = 0; st < nst; ++st) {
    asm volatile("cp.async.wait_group %0;" ::"n"(GP_STAGES - 2) : "memory");
    __syncthreads();  // stage st visible to all; stage st - 1's buffer is free for the copy below
    if (st + GP_STAGES - 1 < nst) issue(st + GP_STAGES - 1);
    asm volatile("cp.async.commit_group;" ::: "memory");
    const double* sA = gsm + (size_t)(st % GP_STAGES) * GP_STAGE_DOUBLES;
    const double* sB = sA + GT * GP_KPAD;
    const int kbase = r0 + st * GP_KS;
#pragma unroll
    for (int kk = 0; kk < GP_KS; kk += 8) {
      double wa = 1.0, wb = 1.0;
      if (w) {
        const int ka = kbase + kk + fk, kb = ka + 4;
        wa = ka < r1 ? __ldg(w + ka) : 0.0;
        wb = kb < r1 ? __ldg(w + kb) : 0.0;
      }
      double af[2][4], bf[8][2];
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        const int r = 32 * wm + 16 * a + fr;
        af[a][0] = wa * sA[r * GP_KPAD + kk + fk];
        af[a][1] = wa * sA[(r + 8) * GP_KPAD + kk + fk];
        af[a][2] = wb * sA[r * GP_KPAD + kk + fk + 4];
        af[a][3] = wb * sA[(r + 8) * GP_KPAD + kk + fk + 4];
      }
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int c = 64 * wn + 8 * b + fr;
        bf[b][0] = sB[c * GP_KPAD + kk + fk];
        bf[b][1] = sB[c * GP_KPAD + kk + fk + 4];
      }
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) dmma16(acc[a][b], af[a], bf[b]);
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
#pragma unroll
  for (int a = 0; a < 2; ++a) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = i0 + 32 * wm + 16 * a + 8 * h + fr;
      if (i >= p) continue;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int j = j0 + 64 * wn + 8 * b + 2 * fk + e;
          if (j >= q) continue;
          if (upper_only && i > j) continue;
          double* dst = C + (long long)j * ldc + i;
          const double v = alpha * acc[a][b][2 * h + e];
          if (atomic)
            atomicAdd(dst, v);
          else
            *dst += v;
        }
      }
    }
  }
}

// Whether gram_pipe_kernel can stage A and B (16-byte copies: aligned bases, even leading dimensions).
inline bool gram_pipe_ok(const double* A, long long lda, const double* B, long long ldb) {
  return (reinterpret_cast<uintptr_t>(A) % 16 == 0) && (reinterpret_cast<uintptr_t>(B) % 16 == 0) && lda % 2 == 0 &&
         ldb % 2 == 0;
}

// Launch of the FP64 Gram tiles (pipelined when the operands allow it), grid (tp, tq, splits).
int launch_gram64(db200_context* ctx, dim3 grid, int n, int p, int q, const double* A, long long lda, const double* B,
                  long long ldb, const double* w, double alpha, double* C, int ldc, int rows, bool upper_only,
                  bool atomic) {
  if (gram_pipe_ok(A, lda, B, ldb)) {
    DB200_CUDA(ctx, cudaFuncSetAttribute(gram_pipe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)GP_SMEM));
    gram_pipe_kernel<<<grid, GTHREADS, GP_SMEM, ctx->stream>>>(n, p, q, A, lda, B, ldb, w, alpha, C, ldc, rows,
                                                               upper_only ? 1 : 0, atomic ? 1 : 0);
  } else {
    gram_kernel<double, double><<<grid, GTHREADS, 0, ctx->stream>>>(n, p, q, A, lda, B, ldb, w, alpha, C, ldc, rows,
                                                                    upper_only ? 1 : 0, atomic ? 1 : 0);
  }
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

// C[n x q] = alpha * A[n x p] * op(B) + beta * C (op(B) = B, p x q, or B^T with B q x p when transB) on the FP64
// tensor cores: one 128 x 128 tile of C per CTA with the whole reduction over p inside it, the warp layout and
// m16n8k8 fragments of gram_kernel.  Stages of 8 columns of A (128 contiguous rows each, one coalesced 256-byte
// read per warp and column) and 8 rows of op(B) are fetched into registers one stage ahead and parked k-major in
// a double-buffered shared tile.
template <typename TA, typename TC>
__global__ void __launch_bounds__(GTHREADS, 1) tall_kernel(int n, int p, int q, const TA* __restrict__ A, long long lda,
                                                           const double* __restrict__ B, int ldb, int transB,
                                                           double alpha, double beta, TC* C, long long ldc) {
  const int i0 = blockIdx.x * GT, j0 = blockIdx.y * GT;
  __shared__ __align__(16) double sA[2][GK][GPAD];
  __shared__ __align__(16) double sB[2][GK][GPAD];
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  const int wm = warp / 2, wn = warp % 2;
  const int fr = lane / 4, fk = lane % 4;
  double acc[2][8][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[a][b][e] = 0.0;
  // A: column k0 + ak, rows i0 + ar + 32 s.  op(B): row k0 + bk, columns j0 + bj + 32 s (B^T rows are contiguous
  // in j, B's columns contiguous in k: consecutive threads walk the contiguous index either way).
  const int ak = threadIdx.x / 32, ar = threadIdx.x % 32;
  const int bk = transB ? threadIdx.x / 32 : threadIdx.x % GK;
  const int bj = transB ? threadIdx.x % 32 : threadIdx.x / GK;
  double va[4], vb[4];
  auto fetch = [&](int k0) {
    const int ka = k0 + ak, kb = k0 + bk;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int i = i0 + ar + 32 * s, j = j0 + bj + 32 * s;
      va[s] = (ka < p && i < n) ? ld64(A + (long long)ka * lda + i) : 0.0;
      vb[s] = (kb < p && j < q) ? (transB ? B[(long long)kb * ldb + j] : B[(long long)j * ldb + kb]) : 0.0;
    }
  };
  auto park = [&](int buf) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      sA[buf][ak][ar + 32 * s] = va[s];
      sB[buf][bk][bj + 32 * s] = vb[s];
    }
  };
  int buf = 0;
  fetch(0);
  park(0);
  __syncthreads();
  for (int k0 = 0; k0 < p; k0 += GK) {
    const bool more = k0 + GK < p;
    if (more) fetch(k0 + GK);
    {
      double af[2][4], bf[8][2];
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        const int r = 32 * wm + 16 * a + fr;
        af[a][0] = sA[buf][fk][r];
        af[a][1] = sA[buf][fk][r + 8];
        af[a][2] = sA[buf][fk + 4][r];
        af[a][3] = sA[buf][fk + 4][r + 8];
      }
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int c = 64 * wn + 8 * b + fr;
        bf[b][0] = sB[buf][fk][c];
        bf[b][1] = sB[buf][fk + 4][c];
      }
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) dmma16(acc[a][b], af[a], bf[b]);
    }
    if (more) park(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }
#pragma unroll
  for (int a = 0; a < 2; ++a) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = i0 + 32 * wm + 16 * a + 8 * h + fr;
      if (i >= n) continue;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int j = j0 + 64 * wn + 8 * b + 2 * fk + e;
          if (j >= q) continue;
          TC* dst = C + (long long)j * ldc + i;
          double v = alpha * acc[a][b][2 * h + e];
          if (beta != 0.0) v += beta * (double)*dst;
          *dst = (TC)v;
        }
      }
    }
  }
}

// One block column of the right-looking blocked upper Cholesky: the kb x kb diagonal block (kb <= 64) is factored
// in every CTA (redundantly; 64 steps with one barrier each, the block's elements in registers, only a reciprocal
// of the pivot on the sequential path, the row scaling by 1/sqrt(pivot) done for all rows afterwards), the last CTA
// to have staged the block writes R11 back (zeros below its diagonal), and CTA c >= 1 overwrites the 64 panel
// columns [k0 + kb + 64 (c - 1), +64) with R11^-T A12 by forward substitution (one warp per 8 columns, the
// solution held two rows per lane and broadcast by shuffles).  The write-back waits for nothing: every CTA counts
// itself in `arrivals` after staging A11, and the CTA that arrives last, when every other CTA has read A11, is
// the one that overwrites it (and re-arms the counter for the next launch).  On a non-positive or NaN pivot
// nothing is written, status <- DB200_ERR_NOT_SPD and *bad <- k0 (first failing block).  A block column after a
// failed one writes nothing.  Follows cholesky_factorize (include/lapack_like.h:10-57): potrf of the diagonal
// block, trsm of the panel, syrk of the trailing matrix (the DMMA gram_kernel or syrk_update_kernel launched after
// this one).
__global__ void __launch_bounds__(256) potrf_block_kernel(double* A, int lda, int k0, int kb, int l, int* status,
                                                          int* bad, int* arrivals) {
  __shared__ double rs[64][65];  // staging, then R11 (row-major: rs[i][j] = R[k0 + i][k0 + j])
  __shared__ double rowk[2][64];
  __shared__ double inv[64];
  __shared__ double dsq[64];
  __shared__ int writer;
  const int t = threadIdx.x;
  // stage the diagonal block coalesced (column j contiguous in i)
  for (int e = t; e < 64 * 64; e += 256) {
    const int i = e & 63, j = e >> 6;
    rs[i][j] = (i < kb && j < kb && i <= j) ? A[(long long)(k0 + j) * lda + k0 + i] : 0.0;
  }
  __syncthreads();  // this CTA's reads of A11 are done
  if (t == 0) {
    __threadfence();
    const int before = atomicAdd(arrivals, 1);
    writer = (before == (int)gridDim.x - 1);
    if (writer) *arrivals = 0;  // every CTA has arrived: re-armed for the next launch
  }
  __syncthreads();
  if (*(volatile int*)status) return;  // an earlier block column failed (checked after counting in)
  // Thread t owns column j = t & 63 and the rows rg + 4 q.  The 64 steps run as 16 groups of 4 (a rolled loop, so
  // that the kernel's code stays small: fully unrolled it missed the instruction cache most of the time when it ran
  // between other kernels); the owners of the group's rows 4 kk .. 4 kk + 3 hold them in a[0], and after each
  // group every thread shifts its column down by one row slot (a[q] holds row rg + 4 (q + kk)), so that no register
  // is indexed at run time.
  const int j = t & 63, rg = t >> 6;
  double a[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) a[q] = rs[rg + 4 * q][j];
  bool failed = false;
#pragma unroll 1
  for (int kk = 0; 4 * kk < kb && !failed; ++kk) {
#pragma unroll
    for (int kr = 0; kr < 4; ++kr) {
      const int k = 4 * kk + kr;
      if (k >= kb) break;
      const double own = a[0];  // row k's element of column j for its owners (rg == kr)
      if (rg == kr) rowk[k & 1][j] = own;
      __syncthreads();  // row k published; also orders the staging reads before the first rs write below
      const double piv = rowk[k & 1][k];
      if (!(piv > 0.0)) {  // the same value in every thread: a uniform exit
        failed = true;
        break;
      }
      const double u = 1.0 / piv;
      const double ckj = rowk[k & 1][j] * u;
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int i = rg + 4 * (q + kk);
        if (i > k && i < 64) a[q] -= rowk[k & 1][i] * ckj;  // i > j entries are never read back
      }
      if (rg == kr) rs[k][j] = (j >= k) ? own : 0.0;  // row k as eliminated (pivot at j == k)
    }
#pragma unroll
    for (int q = 0; q < 15; ++q) a[q] = a[q + 1];
    a[15] = 0.0;
  }
  if (failed) {
    if (writer && t == 0 && atomicCAS(status, 0, DB200_ERR_NOT_SPD) == 0) *bad = k0;
    return;
  }
  // R[k][j] = a_kj / sqrt(a_kk), off the sequential path: square roots first, then every row in parallel
  __syncthreads();
  if (t < kb) {
    const double sd = sqrt(rs[t][t]);
    dsq[t] = sd;
    inv[t] = 1.0 / sd;
  }
  __syncthreads();
  for (int e = t; e < kb * 64; e += 256) {
    const int i = e >> 6, jj = e & 63;
    if (jj > i) rs[i][jj] /= dsq[i];
  }
  __syncthreads();
  if (t < kb) rs[t][t] = dsq[t];
  __syncthreads();
  if (writer) {
    for (int e = t; e < kb * 64; e += 256) {
      const int i = e & 63, jj = e >> 6;
      if (i < kb) A[(long long)(k0 + jj) * lda + k0 + i] = (i <= jj) ? rs[i][jj] : 0.0;
    }
  }
  if (blockIdx.x == 0) return;
  // panel: x = R11^-T b for 8 columns per warp; lane holds rows lane and lane + 32
  const int warp = t >> 5, lane = t & 31;
  const int c0 = k0 + kb + (blockIdx.x - 1) * 64 + warp * 8;
  double v[8][2];
#pragma unroll
  for (int cc = 0; cc < 8; ++cc) {
    const bool ok = c0 + cc < l;
    const double* col = A + (long long)(c0 + cc) * lda + k0;
    v[cc][0] = (ok && lane < kb) ? col[lane] : 0.0;
    v[cc][1] = (ok && lane + 32 < kb) ? col[lane + 32] : 0.0;
  }
  // rows 0..31 of the solution (held in v[.][0]), then rows 32..63 (v[.][1]): two rolled loops, each with constant
  // register indices
#pragma unroll 4
  for (int i = 0; i < 32; ++i) {
    if (i >= kb) break;
    const double ri = inv[i];
    const double r0 = rs[i][lane], r1 = rs[i][lane + 32];  // R[i][row] for this lane's two rows
#pragma unroll
    for (int cc = 0; cc < 8; ++cc) {
      const double x = __shfl_sync(0xffffffffu, v[cc][0], i) * ri;
      if (lane == i) v[cc][0] = x;
      if (lane > i) v[cc][0] -= r0 * x;
      v[cc][1] -= r1 * x;  // lane + 32 > i for every lane
    }
  }
#pragma unroll 4
  for (int i = 32; i < 64; ++i) {
    if (i >= kb) break;
    const double ri = inv[i];
    const double r1 = rs[i][lane + 32];
#pragma unroll
    for (int cc = 0; cc < 8; ++cc) {
      const double x = __shfl_sync(0xffffffffu, v[cc][1], i - 32) * ri;
      if (lane == i - 32) v[cc][1] = x;
      if (lane + 32 > i) v[cc][1] -= r1 * x;
    }
  }
#pragma unroll
  for (int cc = 0; cc < 8; ++cc) {
    if (c0 + cc >= l) continue;
    double* col = A + (long long)(c0 + cc) * lda + k0;
    if (lane < kb) col[lane] = v[cc][0];
    if (lane + 32 < kb) col[lane + 32] = v[cc][1];
  }
}

// Trailing update of the blocked Cholesky: C[m x m] (upper triangle) -= P^T P for the kb x m panel P (kb <= 64, the
// rows of R12 just solved).  One 32 x 32 tile of C per CTA (upper tiles only) so that the few hundred tiles of an
// r ~ 500..4000 factor spread over the whole GPU; the two 64 x 32 panel slices sit in shared memory and each of the
// 256 threads forms 4 outputs with 64-long FP64 dot products.
__global__ void __launch_bounds__(256) syrk_update_kernel(const double* __restrict__ P, int ldp, int kb, int m,
                                                          double* C, int ldc, const int* status) {
  if (*(volatile const int*)status) return;
  int idx = blockIdx.x, bi = 0;
  const int nt = (m + 31) / 32;
  while (idx >= nt - bi) {  // upper tile pairs (bi <= bj), row by row
    idx -= nt - bi;
    ++bi;
  }
  const int bj = bi + idx;
  const int i0 = bi * 32, j0 = bj * 32;
  __shared__ double pi[64][33], pj[64][33];
  for (int e = threadIdx.x; e < 64 * 32; e += 256) {
    const int k = e & 63, c = e >> 6;  // consecutive threads walk k: one column of P is contiguous
    pi[k][c] = (k < kb && i0 + c < m) ? P[(long long)(i0 + c) * ldp + k] : 0.0;
    pj[k][c] = (k < kb && j0 + c < m) ? P[(long long)(j0 + c) * ldp + k] : 0.0;
  }
  __syncthreads();
  const int ti = threadIdx.x & 31, tj = threadIdx.x >> 5;  // rows ti; columns tj + 8 b
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
  for (int k = 0; k < 64; ++k) {
    const double a = pi[k][ti];
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[b] = fma(a, pj[k][tj + 8 * b], acc[b]);
  }
  const int i = i0 + ti;
  if (i >= m) return;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int j = j0 + tj + 8 * b;
    if (j < m && i <= j) C[(long long)j * ldc + i] -= acc[b];
  }
}

// Zero the strictly lower triangle of an l x l matrix.
__global__ void zero_lower_kernel(double* A, int lda, int l) {
  const long long total = (long long)l * l;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % l), j = (int)(e / l);
    if (i > j) A[(long long)j * lda + i] = 0.0;
  }
}

// X = R^-1 for upper triangular R (l x l): one warp per column j solves R x = e_j by column-oriented
// back substitution.
__global__ void trinv_upper_kernel(const double* R, int ldr, int l, double* X, int ldx) {
  const int warps = blockDim.x / 32;
  const int j = blockIdx.x * warps + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (j >= l) return;
  double* x = X + (long long)j * ldx;
  for (int i = lane; i < l; i += 32) x[i] = (i == j) ? 1.0 : 0.0;
  __syncwarp();
  for (int i = j; i >= 0; --i) {
    const double xi = x[i] / R[(long long)i * ldr + i];
    __syncwarp();
    if (lane == 0) x[i] = xi;
    const double* ri = R + (long long)i * ldr;
    for (int k = lane; k < i; k += 32) x[k] -= ri[k] * xi;
    __syncwarp();
  }
}

// Single-CTA triangular solves with an upper factor R (and its transpose L = R^T stored separately so every
// inner product reads a contiguous column):
//   mode 0: solve R^T y = b   (forward; row i of R^T = column i of R)
//   mode 1: solve R x = y     (backward; row i of R = column i of L)
// x/b in place, FP64, x staged in shared memory (l <= 4096).  Blocks of 32 rows: the 16 warps form the off-block
// inner products (two rows each; the coefficients of the nearest 256 columns are loaded before the block's
// barrier, overlapping the previous block's triangle), then warp 0 solves the 32 x 32 triangle from registers it
// also loaded before the barrier (so the 32 sequential steps carry no memory latency), with the diagonal applied
// as a reciprocal computed once per block.  Follows triangular_solve (include/blas_like.h:96-140) for one column.
__global__ void __launch_bounds__(512) trsv_kernel(const double* R, const double* L, int ld, int l, double* x,
                                                   int mode) {
  __shared__ double xs[4096];
  __shared__ double part[32];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  for (int i = threadIdx.x; i < l; i += blockDim.x) xs[i] = x[i];
  const int nb = (l + 31) / 32;
  const double* T = (mode == 0) ? R : L;  // column i0 + lane of T holds this lane's triangle coefficients
  for (int bb = 0; bb < nb; ++bb) {
    const int blk = (mode == 0) ? bb : nb - 1 - bb;
    const int i0 = blk * 32;
    const int bl = min(32, l - i0);
    double tri[32];
    double dinv = 0.0;
    if (warp == 0) {
      const double* c = T + (long long)(i0 + lane) * ld + i0;
#pragma unroll
      for (int r = 0; r < 32; ++r) tri[r] = (lane < bl && r < bl) ? c[r] : 0.0;
    }
    // off-block coefficients of rows i0 + warp and i0 + warp + 16: the nearest 32 PF (= 256) columns are loaded
    // into registers before the barrier (they do not depend on x), so their latency overlaps the previous block's
    // triangle; a longer range finishes in the loop after the barrier
    constexpr int PF = 8;
    double pf[2][PF];
    int kbeg[2], kend[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = i0 + warp + 16 * h;
      kbeg[h] = (mode == 0) ? 0 : i0 + 32;
      kend[h] = (i < l) ? ((mode == 0) ? i0 : l) : kbeg[h];
      // mode 0 reads the columns just below i0 first (nearest the diagonal), mode 1 those just after i0 + 32
      const double* col = T + (long long)(i < l ? i : 0) * ld;
#pragma unroll
      for (int u = 0; u < PF; ++u) {
        const int k = (mode == 0) ? kend[h] - 1 - lane - 32 * u : kbeg[h] + lane + 32 * u;
        pf[h][u] = (k >= kbeg[h] && k < kend[h]) ? col[k] : 0.0;
      }
    }
    __syncthreads();  // xs of the previous block (and the initial staging) visible
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = i0 + warp + 16 * h;
      double s0 = 0.0, s1 = 0.0;
#pragma unroll
      for (int u = 0; u < PF; ++u) {
        const int k = (mode == 0) ? kend[h] - 1 - lane - 32 * u : kbeg[h] + lane + 32 * u;
        if (k >= kbeg[h] && k < kend[h]) {
          if (u & 1)
            s1 += pf[h][u] * xs[k];
          else
            s0 += pf[h][u] * xs[k];
        }
      }
      if (kend[h] - kbeg[h] > 32 * PF) {
        const double* col = T + (long long)i * ld;
        if (mode == 0) {
          for (int k = kbeg[h] + lane; k < kend[h] - 32 * PF; k += 32) s0 += col[k] * xs[k];
        } else {
          for (int k = kbeg[h] + 32 * PF + lane; k < kend[h]; k += 32) s1 += col[k] * xs[k];
        }
      }
      double sum = s0 + s1;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      if (lane == 0) part[warp + 16 * h] = sum;
    }
    __syncthreads();
    if (warp == 0) {
      double dg = 1.0;
#pragma unroll
      for (int r = 0; r < 32; ++r)
        if (r == lane && lane < bl) dg = tri[r];
      dinv = (lane < bl) ? 1.0 / dg : 0.0;
      double v = (lane < bl) ? xs[i0 + lane] - part[lane] : 0.0;
      if (mode == 0) {
#pragma unroll
        for (int r = 0; r < 32; ++r) {
          const double xr = __shfl_sync(0xffffffffu, v * dinv, r);
          if (lane == r) v = xr;
          if (lane > r) v -= tri[r] * xr;
        }
      } else {
#pragma unroll
        for (int r = 31; r >= 0; --r) {
          const double xr = __shfl_sync(0xffffffffu, v * dinv, r);
          if (lane == r) v = xr;
          if (lane < r) v -= tri[r] * xr;
        }
      }
      if (lane < bl) xs[i0 + lane] = v;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < l; i += blockDim.x) x[i] = xs[i];
}

__global__ void transpose_kernel(const double* A, int lda, int m, int n, double* B, int ldb) {
  __shared__ double t[32][33];
  const int bi = blockIdx.x * 32, bj = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = bi + threadIdx.x, j = bj + r;
    if (i < m && j < n) t[r][threadIdx.x] = A[(long long)j * lda + i];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = bj + threadIdx.x, i = bi + r;
    if (i < m && j < n) B[(long long)i * ldb + j] = t[threadIdx.x][r];
  }
}

__global__ void scale_kernel(double* C, int ldc, int m, int n, double beta, int upper_only) {
  const long long total = (long long)m * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % m), j = (int)(e / m);
    if (upper_only && i > j) continue;
    double* p = C + (long long)j * ldc + i;
    *p = (beta == 0.0) ? 0.0 : beta * *p;
  }
}

__global__ void symmetrize_kernel(double* C, int ldc, int l, double shift) {
  // C <- (C + C^T)/2 + shift I, full matrix
  const long long total = (long long)l * l;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % l), j = (int)(e / l);
    if (i > j) continue;
    double* a = C + (long long)j * ldc + i;
    double* b = C + (long long)i * ldc + j;
    double v = 0.5 * (*a + *b);
    if (i == j) v += shift;
    *a = v;
    *b = v;
  }
}

__global__ void fill_upper_from_lower_kernel(double* C, int ldc, int l) {
  const long long total = (long long)l * l;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % l), j = (int)(e / l);
    if (i > j) C[(long long)j * ldc + i] = C[(long long)i * ldc + j];
  }
}

template <typename TS, typename TD>
__global__ void convert_kernel(const TS* src, long long lds, TD* dst, long long ldd, int m, int n) {
  const long long total = (long long)m * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % m), j = (int)(e / m);
    dst[j * ldd + i] = (TD)src[j * lds + i];
  }
}

// C (float) = alpha * T (double) + beta * C
__global__ void axpby_f32_kernel(float* C, long long ldc, const double* T, long long ldt, int m, int n, double alpha,
                                 double beta) {
  const long long total = (long long)m * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % m), j = (int)(e / m);
    float* c = C + j * ldc + i;
    double v = alpha * T[j * ldt + i];
    if (beta != 0.0) v += beta * (double)*c;
    *c = (float)v;
  }
}

// out[0] += sum of squares of the m x n float block
__global__ void sumsq_f32_kernel(const float* A, long long lda, int m, int n, double* out) {
  double s = 0.0;
  const long long total = (long long)m * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const double v = A[(e / m) * lda + (e % m)];
    s = fma(v, v, s);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double w[32];
  if (threadIdx.x % 32 == 0) w[threadIdx.x / 32] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x / 32); ++k) t += w[k];
    atomicAdd(out, t);
  }
}

// FP64 kernel block from a Gram block: K[i + j*ldk] = yi_i yj_j exp(-gamma max(si_i + sj_j - 2 G, 0)) in place
// (G = Xi^T Xj formed by the FP64 Gram kernel); the comparator arithmetic of include/dkernel.cu:116-129 in FP64.
__global__ void rbf_from_gram_f64_kernel(double* K, long long ldk, int m, int n, const double* si, const double* sj,
                                         const float* yi, const float* yj, double gamma) {
  const long long total = (long long)m * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % m), j = (int)(e / m);
    double* k = K + j * ldk + i;
    const double d2 = fmax(si[i] + sj[j] - 2.0 * *k, 0.0);
    double v = exp(-gamma * d2);
    if (yi) v *= (double)yi[i];
    if (yj) v *= (double)yj[j];
    *k = v;
  }
}

// s_i = sum_k x_ik^2 in FP64 for point-major X (d x n, ldx): vecnorm (include/dkernel.cu:102-114) in FP64
__global__ void rownorm_f64_kernel(const float* X, long long ldx, int n, int d, double* s) {
  const int lane = threadIdx.x % 32;
  const long long warps = (long long)gridDim.x * (blockDim.x / 32);
  for (long long i = blockIdx.x * (long long)(blockDim.x / 32) + threadIdx.x / 32; i < n; i += warps) {
    double acc = 0.0;
    for (int k = lane; k < d; k += 32) {
      const double x = X[i * ldx + k];
      acc = fma(x, x, acc);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) s[i] = acc;
  }
}

// Sort v[0..n) descending in place (rank sort, one CTA, n <= 8192).
__global__ void sort_desc_kernel(double* v, int n) {
  extern __shared__ double sv[];
  for (int i = threadIdx.x; i < n; i += blockDim.x) sv[i] = v[i];
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double x = sv[i];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double yj = sv[j];
      rank += (yj > x) || (yj == x && j < i);
    }
    v[rank] = x;
  }
}

__global__ void trace_kernel(const double* C, int ldc, int l, double* out) {
  double s = 0.0;
  for (int i = threadIdx.x; i < l; i += blockDim.x) s += C[(long long)i * ldc + i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double w[32];
  if (threadIdx.x % 32 == 0) w[threadIdx.x / 32] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x / 32); ++k) t += w[k];
    *out = t;
  }
}

// One-sided Jacobi (Hestenes) on the columns of an n x n matrix held in global memory, one CTA: every round
// orthogonalises n/2 disjoint column pairs (round-robin tournament order), one warp per pair.  The singular
// values are the final column norms.  status <- 1 if `max_sweeps` sweeps did not converge.
__global__ void __launch_bounds__(1024) jacobi_svd_kernel(double* A, int lda, int n, int max_sweeps, double tol,
                                                          double* S, int* status) {
  __shared__ unsigned long long worst;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, nw = blockDim.x / 32;
  const int np = (n + 1) & ~1;  // even number of players; index n is a dummy when n is odd
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    if (threadIdx.x == 0) worst = 0ull;
    __syncthreads();
    for (int round = 0; round < np - 1; ++round) {
      for (int k = warp; k < np / 2; k += nw) {
        int p = (k == 0) ? 0 : ((k + round - 1) % (np - 1)) + 1;
        int q = ((np - 1 - k + round - 1) % (np - 1)) + 1;
        if (p >= n || q >= n) continue;
        double* ap = A + (long long)p * lda;
        double* aq = A + (long long)q * lda;
        double al = 0, be = 0, ga = 0;
        for (int i = lane; i < n; i += 32) {
          const double x = ap[i], y = aq[i];
          al = fma(x, x, al);
          be = fma(y, y, be);
          ga = fma(x, y, ga);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          al += __shfl_xor_sync(0xffffffffu, al, o);
          be += __shfl_xor_sync(0xffffffffu, be, o);
          ga += __shfl_xor_sync(0xffffffffu, ga, o);
        }
        const double denom = sqrt(al * be);
        const double ratio = (denom > 0.0) ? fabs(ga) / denom : 0.0;
        if (lane == 0) atomicMax(&worst, (unsigned long long)__double_as_longlong(ratio));
        if (ratio > tol) {
          const double zeta = (be - al) / (2.0 * ga);
          const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
          const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
          for (int i = lane; i < n; i += 32) {
            const double x = ap[i], y = aq[i];
            ap[i] = c * x - s * y;
            aq[i] = s * x + c * y;
          }
        }
      }
      __syncthreads();
    }
    if (__longlong_as_double((long long)worst) <= tol) break;
    __syncthreads();
  }
  for (int p = warp; p < n; p += nw) {
    const double* ap = A + (long long)p * lda;
    double s2 = 0;
    for (int i = lane; i < n; i += 32) s2 = fma(ap[i], ap[i], s2);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    if (lane == 0) S[p] = sqrt(s2);
  }
  if (threadIdx.x == 0) *status = (sweep >= max_sweeps) ? 1 : 0;
}

inline unsigned grid_for(long long total, int threads, int cap) {
  long long b = (total + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (unsigned)b;
}

}  // namespace

template <typename TA, typename TBt>
int gram(db200_context* ctx, int n, int p, int q, const TA* A, long long lda, const TBt* B, long long ldb,
         const double* w, double alpha, double beta, double* C, int ldc, bool upper_only) {
  if (p <= 0 || q <= 0) return DB200_OK;
  scale_kernel<<<grid_for((long long)p * q, 256, 4096), 256, 0, ctx->stream>>>(C, ldc, p, q, beta, upper_only ? 1 : 0);
  count_launch(ctx);
  if (n <= 0) return DB200_OK;
  const int tp = (p + GT - 1) / GT, tq = (q + GT - 1) / GT;
  const int tiles = upper_only ? (tp * (tp + 1)) / 2 : tp * tq;
  // row splits: fill whole waves of one CTA per SM (at least two waves' worth of CTAs)
  int splits = 1;
  {
    const int sms = ctx->num_sms;
    int best = 1;
    double best_eff = -1.0;
    for (int waves = 2; waves <= 8; ++waves) {
      const int sp = (waves * sms) / tiles;
      if (sp < 1) continue;
      const long long ctas = (long long)sp * tiles;
      const double eff = (double)ctas / (double)(((ctas + sms - 1) / sms) * sms);
      if (eff > best_eff + 1e-9) {
        best_eff = eff;
        best = sp;
      }
    }
    splits = best;
  }
  int rows = (n + splits - 1) / splits;
  rows = round_up(rows < GK ? GK : rows, GK);
  splits = (n + rows - 1) / rows;
  if (splits > 65535) return fail(ctx, DB200_ERR_UNSUPPORTED, "gram: too many row splits");
  dim3 grid(tp, tq, splits);
  if constexpr (std::is_same<TA, double>::value && std::is_same<TBt, double>::value)
    return launch_gram64(ctx, grid, n, p, q, A, lda, B, ldb, w, alpha, C, ldc, rows, upper_only, splits > 1);
  gram_kernel<TA, TBt><<<grid, GTHREADS, 0, ctx->stream>>>(n, p, q, A, lda, B, ldb, w, alpha, C, ldc, rows,
                                                     upper_only ? 1 : 0, splits > 1 ? 1 : 0);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

template int gram<float, float>(db200_context*, int, int, int, const float*, long long, const float*, long long,
                                const double*, double, double, double*, int, bool);
template int gram<double, double>(db200_context*, int, int, int, const double*, long long, const double*, long long,
                                  const double*, double, double, double*, int, bool);
template int gram<double, float>(db200_context*, int, int, int, const double*, long long, const float*, long long,
                                 const double*, double, double, double*, int, bool);

template <typename TA, typename TC>
int gemm_tall(db200_context* ctx, int n, int p, int q, const TA* A, long long lda, const double* B, int ldb,
              bool transB, double beta, TC* C, long long ldc, double alpha) {
  if (n <= 0 || q <= 0) return DB200_OK;
  dim3 grid((n + GT - 1) / GT, (q + GT - 1) / GT);
  if (grid.y > 65535) return fail(ctx, DB200_ERR_UNSUPPORTED, "gemm_tall: q too large");
  tall_kernel<TA, TC><<<grid, GTHREADS, 0, ctx->stream>>>(n, p, q, A, lda, B, ldb, transB ? 1 : 0, alpha, beta, C,
                                                          ldc);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

template int gemm_tall<float, double>(db200_context*, int, int, int, const float*, long long, const double*, int,
                                      bool, double, double*, long long, double);
template int gemm_tall<double, double>(db200_context*, int, int, int, const double*, long long, const double*, int,
                                       bool, double, double*, long long, double);
template int gemm_tall<double, float>(db200_context*, int, int, int, const double*, long long, const double*, int,
                                      bool, double, float*, long long, double);
template int gemm_tall<float, float>(db200_context*, int, int, int, const float*, long long, const double*, int,
                                     bool, double, float*, long long, double);

int potrf_upper(db200_context* ctx, double* A, int lda, int l, int* d_status, int* d_bad, int nb) {
  if (nb < 1 || nb > 64) nb = 64;
  // up to l = 544 (the barrier's capacity matrices, the CholeskyQR2 and Nystrom Grams) the whole factor is one
  // launch on a thread-block cluster; an explicit smaller block size keeps the multi-kernel path
  if (nb == 64) {
    const int s = potrf_cluster(ctx, A, lda, l, d_status, d_bad);
    if (s != DB200_ERR_UNSUPPORTED) return s;
  }
  // the diagonal-block kernel's arrival counter starts every factorisation at zero
  DB200_CUDA(ctx, cudaMemsetAsync(ctx->d_status + 1, 0, sizeof(int), ctx->stream));
  // A trailing matrix of at least one wave of 128 x 128 upper tiles takes its update on the FP64 tensor cores
  // (gram_kernel, alpha = -1, added in place).  While the matrix beyond the next 8 nb columns is that large, the
  // factor goes by outer panels of 8 nb columns: each nb-block of the panel is factored (potrf_block_kernel, which
  // also solves its row to the last column), the panel's own later rows are updated at once (a strip of at most
  // 7 nb rows), and the trailing matrix takes one rank-8 nb update per panel instead of eight rank-nb ones
  // (measured at n = 16384 / 32768 with nb = 64: rank-64 updates 225 ms / -, rank-256 120 / 856 ms, rank-512
  // 105 / 755 ms).
  auto big = [&](int rest) {
    const int tp = (rest + GT - 1) / GT;
    return rest > 0 && tp * (tp + 1) / 2 >= ctx->num_sms;
  };
  for (int K0 = 0; K0 < l;) {
    const int rest0 = l - K0;
    const int KB = big(rest0 - 8 * nb) ? 8 * nb : (rest0 < nb ? rest0 : nb);
    for (int k0 = K0; k0 < K0 + KB; k0 += nb) {
      const int kb = (K0 + KB - k0 < nb) ? K0 + KB - k0 : nb;
      const int rest = l - k0 - kb;
      potrf_block_kernel<<<1 + (rest + 63) / 64, 256, 0, ctx->stream>>>(A, lda, k0, kb, l, d_status, d_bad,
                                                                         ctx->d_status + 1);
      count_launch(ctx);
      const int pr = K0 + KB - (k0 + kb);  // rows of this panel below the block
      if (pr > 0) {
        const double* P = A + (long long)(k0 + kb) * lda + k0;
        double* C = A + (long long)(k0 + kb) * lda + k0 + kb;
        const int s2 = launch_gram64(ctx, dim3((pr + GT - 1) / GT, (rest + GT - 1) / GT, 1), kb, pr, rest, P, lda, P,
                                     lda, nullptr, -1.0, C, lda, kb, true, false);
        if (s2) return s2;
      }
    }
    const int rest = l - K0 - KB;
    if (rest > 0) {
      // trailing update A22 -= A12^T A12 (upper triangle only) with the panel's KB rows
      const double* P = A + (long long)(K0 + KB) * lda + K0;
      double* C = A + (long long)(K0 + KB) * lda + K0 + KB;
      if (KB > nb || big(rest)) {
        const int tp = (rest + GT - 1) / GT;
        const int s2 = launch_gram64(ctx, dim3(tp, tp, 1), KB, rest, rest, P, lda, P, lda, nullptr, -1.0, C, lda, KB,
                                     true, false);
        if (s2) return s2;
      } else {
        // the r ~ 500..2000 capacity factors of the barrier: 32 x 32 tiles, so that they spread over the GPU
        const int nt = (rest + 31) / 32;
        syrk_update_kernel<<<nt * (nt + 1) / 2, 256, 0, ctx->stream>>>(P, lda, KB, rest, C, lda, d_status);
        count_launch(ctx);
      }
    }
    K0 += KB;
  }
  zero_lower_kernel<<<grid_for((long long)l * l, 256, 1024), 256, 0, ctx->stream>>>(A, lda, l);
  count_launch(ctx);
  DB200_CUDA(ctx, cudaGetLastError());
  return DB200_OK;
}

int trinv_upper(db200_context* ctx, const double* R, int ldr, int l, double* X, int ldx) {
  trinv_upper_kernel<<<(l + 7) / 8, 256, 0, ctx->stream>>>(R, ldr, l, X, ldx);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int trsv_upper(db200_context* ctx, const double* R, const double* L, int ld, int l, double* x, bool transposed) {
  if (l > 4096) return fail(ctx, DB200_ERR_UNSUPPORTED, "trsv: l > 4096");
  trsv_kernel<<<1, 512, 0, ctx->stream>>>(R, L, ld, l, x, transposed ? 0 : 1);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int transpose64(db200_context* ctx, const double* A, int lda, int m, int n, double* B, int ldb) {
  dim3 grid((m + 31) / 32, (n + 31) / 32), block(32, 8);
  transpose_kernel<<<grid, block, 0, ctx->stream>>>(A, lda, m, n, B, ldb);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int symmetrize(db200_context* ctx, double* C, int ldc, int l, double shift) {
  symmetrize_kernel<<<grid_for((long long)l * l, 256, 1024), 256, 0, ctx->stream>>>(C, ldc, l, shift);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int mirror_upper(db200_context* ctx, double* C, int ldc, int l) {
  fill_upper_from_lower_kernel<<<grid_for((long long)l * l, 256, 1024), 256, 0, ctx->stream>>>(C, ldc, l);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

template <typename TS, typename TD>
int convert(db200_context* ctx, const TS* src, long long lds, TD* dst, long long ldd, int m, int n) {
  convert_kernel<TS, TD><<<grid_for((long long)m * n, 256, 8 * ctx->num_sms), 256, 0, ctx->stream>>>(src, lds, dst,
                                                                                                     ldd, m, n);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}
template int convert<double, float>(db200_context*, const double*, long long, float*, long long, int, int);
template int convert<float, double>(db200_context*, const float*, long long, double*, long long, int, int);
template int convert<double, double>(db200_context*, const double*, long long, double*, long long, int, int);
template int convert<float, float>(db200_context*, const float*, long long, float*, long long, int, int);

int jacobi_svd_values(db200_context* ctx, double* A, int lda, int n, double* S, int* d_status) {
  jacobi_svd_kernel<<<1, 1024, 0, ctx->stream>>>(A, lda, n, 40, 1e-15, S, d_status);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int axpby_f32(db200_context* ctx, float* C, long long ldc, const double* T, long long ldt, int m, int n,
              double alpha, double beta) {
  axpby_f32_kernel<<<grid_for((long long)m * n, 256, 8 * ctx->num_sms), 256, 0, ctx->stream>>>(C, ldc, T, ldt, m, n,
                                                                                                alpha, beta);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int sumsq_f32(db200_context* ctx, const float* A, long long lda, int m, int n, double* d_out) {
  sumsq_f32_kernel<<<grid_for((long long)m * n, 256, 8 * ctx->num_sms), 256, 0, ctx->stream>>>(A, lda, m, n, d_out);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int rbf_from_gram_f64(db200_context* ctx, double* K, long long ldk, int m, int n, const double* si, const double* sj,
                      const float* yi, const float* yj, double gamma) {
  rbf_from_gram_f64_kernel<<<grid_for((long long)m * n, 256, 16 * ctx->num_sms), 256, 0, ctx->stream>>>(
      K, ldk, m, n, si, sj, yi, yj, gamma);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int rownorm_f64(db200_context* ctx, const float* X, long long ldx, int n, int d, double* s) {
  rownorm_f64_kernel<<<grid_for((long long)n * 32, 256, 16 * ctx->num_sms), 256, 0, ctx->stream>>>(X, ldx, n, d, s);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int sort_desc(db200_context* ctx, double* v, int n) {
  if (n > 8192) return fail(ctx, DB200_ERR_UNSUPPORTED, "sort_desc: n > 8192");
  sort_desc_kernel<<<1, 1024, sizeof(double) * n, ctx->stream>>>(v, n);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int trace(db200_context* ctx, const double* C, int ldc, int l, double* d_out) {
  trace_kernel<<<1, 1024, 0, ctx->stream>>>(C, ldc, l, d_out);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

}  // namespace db200
