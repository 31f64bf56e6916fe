// LU factorisation with partial pivoting on the GPU (FP32, column major): the reference's
// lu_factorize_partial_pivot / lu_factorize_partial_pivot_replicate_panel / lu_factorize_no_pivot
// (include/lapack_like.h:93-279) for a matrix in device memory.
//
// Blocked right-looking, panels of W = 32 columns:
//   lu_panel_kernel   one CTA factors the m x w panel column by column: argmax |a| below the diagonal (first
//                     index on ties, as the reference's scan and LAPACK's isamax), row swap inside the panel,
//                     scaling by the reciprocal pivot (as the reference's inv_pivot), rank-1 update of the
//                     panel's remaining columns
//   lu_laswp_kernel   the panel's row interchanges applied in order to the other columns (one thread per column)
//   lu_trsm_kernel    U12 = L11^-1 A12 with the unit lower w x w block in shared memory (one thread per column)
//   lu_update_kernel  A22 -= L21 U12: 64 x 64 output tiles, K = w, FP32 FMA
// Pivots are recorded 1-based relative to the first row, like LAPACK's ipiv and the reference's.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>

#include "internal.h"

namespace db200 {

namespace {

constexpr int W = 32;            // panel width
constexpr int PANEL_THREADS = 1024;
constexpr int UT = 64;           // update tile (rows and columns)

__global__ void __launch_bounds__(PANEL_THREADS) lu_panel_kernel(float* A, long long lda, int m, int k, int w,
                                                                int* ipiv, int pivot, int* singular) {
  __shared__ float red_v[PANEL_THREADS / 32];
  __shared__ int red_i[PANEL_THREADS / 32];
  __shared__ float urow[W];
  __shared__ int piv_row;
  const int tid = threadIdx.x, lane = tid % 32, wid = tid / 32;
  for (int jj = 0; jj < w; ++jj) {
    const int j = k + jj;
    float* col = A + (long long)j * lda;
    if (pivot) {
      // argmax |A[r, j]| over r in [j, m): the largest value, the smallest row among equal values
      float bv = -1.0f;
      int bi = m;
      for (int r = j + tid; r < m; r += PANEL_THREADS) {
        const float v = fabsf(col[r]);
        if (v > bv) {
          bv = v;
          bi = r;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) {
          bv = ov;
          bi = oi;
        }
      }
      if (lane == 0) {
        red_v[wid] = bv;
        red_i[wid] = bi;
      }
      __syncthreads();
      if (wid == 0) {
        bv = red_v[lane];
        bi = red_i[lane];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
          const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
          if (ov > bv || (ov == bv && oi < bi)) {
            bv = ov;
            bi = oi;
          }
        }
        if (lane == 0) {
          piv_row = bi < m ? bi : j;
          ipiv[j] = piv_row + 1;
        }
      }
      __syncthreads();
      const int p = piv_row;
      if (p != j && tid < w) {  // swap rows j and p inside the panel
        float* c = A + (long long)(k + tid) * lda;
        const float t = c[j];
        c[j] = c[p];
        c[p] = t;
      }
    } else if (tid == 0) {
      ipiv[j] = j + 1;
    }
    __syncthreads();
    if (tid < w - jj - 1) urow[tid] = A[j + (long long)(j + 1 + tid) * lda];  // row j right of the diagonal
    const float d = col[j];
    __syncthreads();
    if (d == 0.0f) {
      if (tid == 0) atomicCAS(singular, 0, j + 1);
      continue;  // nothing to eliminate with: leave the column as it is
    }
    const float inv = 1.0f / d;
    const int rest = w - jj - 1;
    // Scale and update RU rows per thread at a time, the loads of 8 columns issued before their FMAs: the panel
    // lives in L2, so the kernel is bound by how many loads each thread keeps in flight.
    constexpr int RU = 4;
    for (int r0 = j + 1 + tid; r0 < m; r0 += RU * PANEL_THREADS) {
      float l[RU];
#pragma unroll
      for (int u = 0; u < RU; ++u) {
        const int r = r0 + u * PANEL_THREADS;
        l[u] = r < m ? col[r] * inv : 0.0f;
        if (r < m) col[r] = l[u];
      }
      for (int c0 = 0; c0 < rest; c0 += 8) {
        float v[RU][8];
#pragma unroll
        for (int u = 0; u < RU; ++u)
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int r = r0 + u * PANEL_THREADS;
            v[u][q] = (r < m && c0 + q < rest) ? A[r + (long long)(j + 1 + c0 + q) * lda] : 0.0f;
          }
#pragma unroll
        for (int u = 0; u < RU; ++u)
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int r = r0 + u * PANEL_THREADS;
            if (r < m && c0 + q < rest) A[r + (long long)(j + 1 + c0 + q) * lda] = fmaf(-l[u], urow[c0 + q], v[u][q]);
          }
      }
    }
    __syncthreads();
  }
}

// Row interchanges ipiv[k .. k+w) (1-based, relative to row 0) applied in order to columns [c0, c1) and
// [c2, c3).
__global__ void lu_laswp_kernel(float* A, long long lda, int k, int w, const int* ipiv, int c0, int c1, int c2,
                                int c3) {
  const int n1 = c1 - c0, total = n1 + (c3 - c2);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int c = t < n1 ? c0 + t : c2 + (t - n1);
    float* col = A + (long long)c * lda;
    for (int jj = 0; jj < w; ++jj) {
      const int j = k + jj, p = ipiv[j] - 1;
      if (p != j) {
        const float v = col[j];
        col[j] = col[p];
        col[p] = v;
      }
    }
  }
}

// A[k:k+w, c] = L11^-1 A[k:k+w, c] for c in [c0, c1), L11 unit lower (w x w at A[k, k]).
__global__ void __launch_bounds__(256) lu_trsm_kernel(float* A, long long lda, int k, int w, int c0, int c1) {
  __shared__ float L[W][W + 1];
  for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
    const int r = e % w, c = e / w;
    L[r][c] = A[(k + r) + (long long)(k + c) * lda];
  }
  __syncthreads();
  for (int c = c0 + blockIdx.x * blockDim.x + threadIdx.x; c < c1; c += gridDim.x * blockDim.x) {
    float* col = A + (long long)c * lda + k;
    float x[W];
#pragma unroll
    for (int r = 0; r < W; ++r) x[r] = r < w ? col[r] : 0.0f;
#pragma unroll
    for (int r = 1; r < W; ++r) {
      float s = x[r];
#pragma unroll
      for (int q = 0; q < r; ++q) s = fmaf(-L[r][q], x[q], s);
      x[r] = s;
    }
#pragma unroll
    for (int r = 0; r < W; ++r)
      if (r < w) col[r] = x[r];
  }
}

// A[r0:m, c0:n] -= A[r0:m, k:k+w] A[k:k+w, c0:n]; 64 x 64 tiles, 256 threads, 4 x 4 outputs per thread.
__global__ void __launch_bounds__(256) lu_update_kernel(float* A, long long lda, int m, int n, int k, int w, int r0,
                                                        int c0) {
  __shared__ float Ls[W][UT + 4];  // L21 tile, k-major
  __shared__ float Us[W][UT + 4];  // U12 tile
  const int tr = r0 + blockIdx.y * UT, tc = c0 + blockIdx.x * UT;
  for (int e = threadIdx.x; e < W * UT; e += blockDim.x) {
    const int q = e / UT, i = e % UT;
    Ls[q][i] = (q < w && tr + i < m) ? A[(tr + i) + (long long)(k + q) * lda] : 0.0f;
    const int cq = e % W, cj = e / W;  // U12: row k+cq, column tc+cj (contiguous in q)
    Us[cq][cj] = (cq < w && tc + cj < n) ? A[(k + cq) + (long long)(tc + cj) * lda] : 0.0f;
  }
  __syncthreads();
  // rows are the fast thread index, so each warp reads and writes 16 consecutive rows of 2 columns
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  float acc[4][4] = {};
#pragma unroll 8
  for (int q = 0; q < W; ++q) {
    float a[4], b[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a[u] = Ls[q][tx + 16 * u];
      b[u] = Us[q][ty + 16 * u];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(a[u], b[v], acc[u][v]);
  }
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const int c = tc + ty + 16 * v;
    if (c >= n) continue;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = tr + tx + 16 * u;
      if (r < m) A[r + (long long)c * lda] -= acc[u][v];
    }
  }
}

}  // namespace

int lu_factorize(db200_context* ctx, int m, int n, int nleft, float* A, long long lda, int* ipiv, int pivot,
                 int swap_left_panels) {
  const int mn = m < n ? m : n;
  int* singular = static_cast<int*>(slot_buffer(ctx, SLOT_LA, 256));
  if (!singular) return DB200_ERR_NOMEM;
  DB200_CUDA(ctx, cudaMemsetAsync(singular, 0, sizeof(int), ctx->stream));
  for (int k = 0; k < mn; k += W) {
    const int w = mn - k < W ? mn - k : W;
    lu_panel_kernel<<<1, PANEL_THREADS, 0, ctx->stream>>>(A, lda, m, k, w, ipiv, pivot, singular);
    DB200_CUDA(ctx, cudaGetLastError());
    int launches = 1;
    if (pivot) {
      // columns left of the panel: all of them (the reference's lu_factorize_partial_pivot, the caller's nleft
      // columns included), or none (lu_factorize_partial_pivot_replicate_panel); columns right of it: all
      const int c0 = swap_left_panels ? -nleft : 0, c1 = swap_left_panels ? k : 0;
      const int total = (c1 - c0) + (n - (k + w));
      if (total > 0) {
        const int blocks = (total + 255) / 256;
        lu_laswp_kernel<<<blocks < 4096 ? blocks : 4096, 256, 0, ctx->stream>>>(A, lda, k, w, ipiv, c0, c1, k + w,
                                                                                 n);
        DB200_CUDA(ctx, cudaGetLastError());
        ++launches;
      }
    }
    if (k + w < n) {
      const int cols = n - (k + w);
      const int blocks = (cols + 255) / 256;
      lu_trsm_kernel<<<blocks < 4096 ? blocks : 4096, 256, 0, ctx->stream>>>(A, lda, k, w, k + w, n);
      DB200_CUDA(ctx, cudaGetLastError());
      ++launches;
      if (k + w < m) {
        dim3 grid((unsigned)((cols + UT - 1) / UT), (unsigned)((m - (k + w) + UT - 1) / UT));
        lu_update_kernel<<<grid, 256, 0, ctx->stream>>>(A, lda, m, n, k, w, k + w, k + w);
        DB200_CUDA(ctx, cudaGetLastError());
        ++launches;
      }
    }
    count_launch(ctx, launches);
  }
  int sing = 0;
  DB200_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, singular, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::memcpy(&sing, ctx->h_pinned, sizeof(int));
  if (sing) return fail(ctx, DB200_ERR_SINGULAR, "lu_factorize: zero pivot in column " + std::to_string(sing));
  return DB200_OK;
}

}  // namespace db200

using namespace db200;

extern "C" int db200_lu_factorize(db200_context* ctx, int m, int n, int nleft, float* A, int lda, int* ipiv,
                                  int pivot, int swap_left_panels) {
  if (!ctx) return DB200_ERR_INVALID;
  if (m < 0 || n < 0 || nleft < 0 || lda < (m > 1 ? m : 1) || ((m > 0 && n > 0) && (!A || !ipiv)))
    return fail(ctx, DB200_ERR_INVALID, "db200_lu_factorize: bad arguments");
  if (m == 0 || n == 0) return DB200_OK;
  return lu_factorize(ctx, m, n, nleft, A, lda, ipiv, pivot ? 1 : 0, swap_left_panels ? 1 : 0);
}
