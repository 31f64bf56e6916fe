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
//   lu_update_kernel  A22 -= L21 U12: 64 x 64 output tiles, K = w, FP32 FMA (small trailing matrices)
//   lu_update_tc      the same update on the tcgen05 tile engine (UPDATE mode) once A22 holds a million entries:
//                     the rows of L21 and the columns of U12 as two point sets, each scaled by a power of two and
//                     split into fp16 hi + lo (22 significant bits), hi.hi + hi.lo + lo.hi accumulated in fp32,
//                     A22 read, updated and written once by the epilogue
// Pivots are recorded 1-based relative to the first row, like LAPACK's ipiv and the reference's.
#include <cfloat>
#include <cmath>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "gridsync.cuh"
#include "internal.h"
#include "ptx.cuh"

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

// ------------------------------------------------------------------ cooperative panel
// The panel's rows split over G co-resident CTAs, each holding its slice (R rows x w columns) in shared memory.
// Per column one grid barrier: before it every CTA publishes its best pivot candidate (value, row, the row's w
// values) and the owner of row j publishes row j; after it every CTA picks the same pivot from the G candidates,
// the owners of rows j and p exchange them in shared memory, and every CTA scales and updates its own rows.  The
// published slots alternate between two buffers by column parity: a CTA writes slot (jj & 1) only after the
// barrier of column jj - 1, which every CTA reaches after it has read the slots of column jj - 2.
constexpr int CP_THREADS = 256;
constexpr int CP_MAX_ROWS = 1536;   // rows per CTA held in shared memory (1536 x 32 x 4 B = 192 KB)
constexpr int CAND = W + 2;         // candidate record: |value|, row, the row's W values

__global__ void __launch_bounds__(CP_THREADS) lu_panel_coop_kernel(float* A, long long lda, int m, int k, int w,
                                                                   int R, int* ipiv, int pivot, int* singular,
                                                                   unsigned* bar, unsigned bar_base, float* cand,
                                                                   float* rowj, int* status) {
  extern __shared__ float tile[];  // [W][R]: tile[c * R + i] = A[r0 + i, k + c]
  __shared__ float urow[W];
  __shared__ float red_v[CP_THREADS / 32];
  __shared__ int red_i[CP_THREADS / 32];
  __shared__ int s_win;
  const int tid = threadIdx.x, lane = tid % 32, wid = tid / 32;
  const int G = gridDim.x, b = blockIdx.x;
  const int r0 = k + b * R;
  const int rows = max(0, min(R, m - r0));
  for (int e = tid; e < w * R; e += CP_THREADS) {
    const int c = e / R, i = e % R;
    tile[c * R + i] = i < rows ? A[(r0 + i) + (long long)(k + c) * lda] : 0.0f;
  }
  __syncthreads();
  for (int jj = 0; jj < w; ++jj) {
    const int j = k + jj, par = jj & 1;
    float* my_cand = cand + ((size_t)par * G + b) * CAND;
    // local candidate: the largest |a| of column jj among own rows >= j, the smallest row on ties
    float bv = -1.0f;
    int bi = m;
    for (int i = tid; i < rows; i += CP_THREADS) {
      const int r = r0 + i;
      const float v = fabsf(tile[jj * R + i]);
      if (r >= j && v > bv) {
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
    if (tid == 0) {
      for (int q = 1; q < CP_THREADS / 32; ++q)
        if (red_v[q] > bv || (red_v[q] == bv && red_i[q] < bi)) {
          bv = red_v[q];
          bi = red_i[q];
        }
      my_cand[0] = bv;
      my_cand[1] = __int_as_float(bi);
      s_win = bi;
    }
    __syncthreads();
    const int lbi = s_win;
    if (tid < w) my_cand[2 + tid] = (lbi < m) ? tile[tid * R + (lbi - r0)] : 0.0f;
    if (j >= r0 && j < r0 + rows && tid < w) rowj[par * W + tid] = tile[tid * R + (j - r0)];
    if (!grid_barrier(bar, bar_base + (unsigned)(jj + 1) * (unsigned)G, status, 1, DB200_WAIT_TIMEOUT_NS)) return;
    // the same pivot in every CTA: the largest candidate, the smallest row on ties (one warp scans the G records)
    if (wid == 0) {
      float gv = -1.0f;
      int gb = -1, gi = m;
      for (int q = lane; q < G; q += 32) {
        const float* cq = cand + ((size_t)par * G + q) * CAND;
        const float v = cq[0];
        const int r = __float_as_int(cq[1]);
        if (v > gv || (v == gv && r < gi)) {
          gv = v;
          gi = r;
          gb = q;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, gv, o);
        const int oi = __shfl_xor_sync(0xffffffffu, gi, o);
        const int ob = __shfl_xor_sync(0xffffffffu, gb, o);
        if (ov > gv || (ov == gv && oi < gi)) {
          gv = ov;
          gi = oi;
          gb = ob;
        }
      }
      if (lane == 0) {
        s_win = pivot ? gb : -1;
        if (b == 0) ipiv[j] = (pivot && gi < m) ? gi + 1 : j + 1;
        red_i[0] = (pivot && gi < m) ? gi : j;
      }
    }
    __syncthreads();
    const int p = red_i[0], wb = s_win;
    if (tid < w) {
      const float* src = (wb >= 0 && p != j) ? cand + ((size_t)par * G + wb) * CAND + 2 : rowj + par * W;
      urow[tid] = src[tid];
    }
    __syncthreads();
    if (p != j && tid < w) {
      if (p >= r0 && p < r0 + rows) tile[tid * R + (p - r0)] = rowj[par * W + tid];  // old row j to row p
      if (j >= r0 && j < r0 + rows) tile[tid * R + (j - r0)] = urow[tid];           // pivot row to row j
    }
    __syncthreads();
    const float d = urow[jj];
    if (d == 0.0f) {
      if (b == 0 && tid == 0) atomicCAS(singular, 0, j + 1);
      continue;
    }
    const float inv = 1.0f / d;
    for (int i = tid; i < rows; i += CP_THREADS) {
      if (r0 + i <= j) continue;
      const float l = tile[jj * R + i] * inv;
      tile[jj * R + i] = l;
      for (int c = jj + 1; c < w; ++c) tile[c * R + i] = fmaf(-l, urow[c], tile[c * R + i]);
    }
    __syncthreads();
  }
  for (int e = tid; e < w * R; e += CP_THREADS) {
    const int c = e / R, i = e % R;
    if (i < rows) A[(r0 + i) + (long long)(k + c) * lda] = tile[c * R + i];
  }
}

// ------------------------------------------------------------------ cluster panel
// The same column steps over the G <= 8 CTAs of one thread-block cluster (the grid is that one cluster): each CTA
// holds its slice in shared memory and keeps its candidate record and, when it owns row j, row j in its own shared
// memory (two slots by column parity, as above); one cluster barrier per column replaces the grid barrier, and the
// other CTAs' records are read through distributed shared memory.  The pivot rule and the arithmetic are those of
// lu_panel_coop_kernel, so both give the same factors.
constexpr int CL_MAX = 16;        // cluster size limit (above 8 when the GPU allows non-portable clusters)
constexpr int CL_THREADS = 1024;  // a thread per row of a 1024-row slice: the column step's latency chain is short

__device__ __forceinline__ float ld_cluster_f32(uint32_t cluster_addr) {
  float v;
  asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(cluster_addr) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__global__ void __launch_bounds__(CL_THREADS) lu_panel_cluster_kernel(float* A, long long lda, int m, int k, int w,
                                                                      int R, int* ipiv, int pivot, int* singular) {
  extern __shared__ float tile[];  // [W][R]: tile[c * R + i] = A[r0 + i, k + c]
  __shared__ float s_cand[2][CAND];  // this CTA's candidate record per column parity
  __shared__ float s_rowj[2][W];     // row j, in the CTA that owns it
  __shared__ float urow[W];
  __shared__ float red_v[CL_THREADS / 32];
  __shared__ int red_i[CL_THREADS / 32];
  __shared__ int s_win;
  const int tid = threadIdx.x, lane = tid % 32, wid = tid / 32;
  const int G = gridDim.x, b = blockIdx.x;  // one cluster: the block index is the rank in the cluster
  const int r0 = k + b * R;
  const int rows = max(0, min(R, m - r0));
  for (int e = tid; e < w * R; e += CL_THREADS) {
    const int c = e / R, i = e % R;
    tile[c * R + i] = i < rows ? A[(r0 + i) + (long long)(k + c) * lda] : 0.0f;
  }
  __syncthreads();
  for (int jj = 0; jj < w; ++jj) {
    const int j = k + jj, par = jj & 1;
    // local candidate: the largest |a| of column jj among own rows >= j, the smallest row on ties
    float bv = -1.0f;
    int bi = m;
    for (int i = tid; i < rows; i += CL_THREADS) {
      const int r = r0 + i;
      const float v = fabsf(tile[jj * R + i]);
      if (r >= j && v > bv) {
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
    if (wid == 0) {  // the 32 warp candidates, reduced by one warp (lower warps hold lower rows: ties keep the row)
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
        s_cand[par][0] = bv;
        s_cand[par][1] = __int_as_float(bi);
        s_win = bi;
      }
    }
    __syncthreads();
    const int lbi = s_win;
    if (tid < w) s_cand[par][2 + tid] = (lbi < m) ? tile[tid * R + (lbi - r0)] : 0.0f;
    if (j >= r0 && j < r0 + rows && tid < w) s_rowj[par][tid] = tile[tid * R + (j - r0)];
    cluster_sync_all();  // every record of this column published
    // the same pivot in every CTA: the largest candidate, the smallest row on ties (one warp reads the G records)
    if (wid == 0) {
      float gv = -1.0f;
      int gb = -1, gi = m;
      for (int q = lane; q < G; q += 32) {
        const uint32_t cq = mapa_shared(smem_addr(&s_cand[par][0]), (uint32_t)q);
        const float v = ld_cluster_f32(cq);
        const int r = __float_as_int(ld_cluster_f32(cq + 4));
        if (v > gv || (v == gv && r < gi)) {
          gv = v;
          gi = r;
          gb = q;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, gv, o);
        const int oi = __shfl_xor_sync(0xffffffffu, gi, o);
        const int ob = __shfl_xor_sync(0xffffffffu, gb, o);
        if (ov > gv || (ov == gv && oi < gi)) {
          gv = ov;
          gi = oi;
          gb = ob;
        }
      }
      if (lane == 0) {
        s_win = pivot ? gb : -1;
        if (b == 0) ipiv[j] = (pivot && gi < m) ? gi + 1 : j + 1;
        red_i[0] = (pivot && gi < m) ? gi : j;
      }
    }
    __syncthreads();
    const int p = red_i[0], wb = s_win;
    const uint32_t owner_j = (uint32_t)((j - k) / R);
    float old_j = 0.0f;  // row j's value in column tid, from its owner
    if (tid < w) {
      old_j = ld_cluster_f32(mapa_shared(smem_addr(&s_rowj[par][tid]), owner_j));
      urow[tid] = (wb >= 0 && p != j) ? ld_cluster_f32(mapa_shared(smem_addr(&s_cand[par][2 + tid]), (uint32_t)wb))
                                      : old_j;
    }
    __syncthreads();
    if (p != j && tid < w) {
      if (p >= r0 && p < r0 + rows) tile[tid * R + (p - r0)] = old_j;      // old row j to row p
      if (j >= r0 && j < r0 + rows) tile[tid * R + (j - r0)] = urow[tid];  // pivot row to row j
    }
    __syncthreads();
    const float d = urow[jj];
    if (d == 0.0f) {  // the same in every CTA: all of them go on to the next column's cluster barrier
      if (b == 0 && tid == 0) atomicCAS(singular, 0, j + 1);
      continue;
    }
    const float inv = 1.0f / d;
    for (int i = tid; i < rows; i += CL_THREADS) {
      if (r0 + i <= j) continue;
      const float l = tile[jj * R + i] * inv;
      tile[jj * R + i] = l;
      for (int c = jj + 1; c < w; ++c) tile[c * R + i] = fmaf(-l, urow[c], tile[c * R + i]);
    }
    __syncthreads();
  }
  cluster_sync_all();  // no CTA leaves while another may still read its records
  for (int e = tid; e < w * R; e += CL_THREADS) {
    const int c = e / R, i = e % R;
    if (i < rows) A[(r0 + i) + (long long)(k + c) * lda] = tile[c * R + i];
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

// Workspace bytes of lu_update_tc for a trailing matrix of `rows` x `cols`.
size_t lu_update_tc_bytes(int rows, int cols) {
  const size_t per_point = 2 * 32 * 2;  // fp16 hi | lo of 32 features
  return 4096 + (size_t)point_pad(rows) * per_point + packed_norm_floats(point_pad(rows)) * 4 +
         (size_t)point_pad(cols) * per_point + packed_norm_floats(point_pad(cols)) * 4;
}

int lu_update_tc(db200_context* ctx, float* A, long long lda, int m, int n, int k, int w, int r0, int c0, void* ws) {
  const int rows = m - r0, cols = n - c0, dp = 32;
  Carve cv{static_cast<char*>(ws)};
  PackedPoints pl;  // L21: point i = row r0 + i, features A[r0 + i, k .. k + w) (column major: feature-major)
  pl.n = rows;
  pl.npad = point_pad(rows);
  pl.dp = dp;
  void* xl = cv.take<uint16_t>((size_t)pl.npad * 2 * dp);
  float* nl = cv.take<float>(packed_norm_floats(pl.npad));
  int st = pack_points(ctx, A + r0 + (long long)k * lda, (int)lda, DB200_FEATURE_MAJOR, rows, w, dp, pl.npad, xl, nl);
  if (st) return st;
  pl.xp = xl;
  pl.norms = nl;
  PackedPoints pu;  // U12: point j = column c0 + j, features A[k .. k + w, c0 + j] (point-major)
  pu.n = cols;
  pu.npad = point_pad(cols);
  pu.dp = dp;
  void* xu = cv.take<uint16_t>((size_t)pu.npad * 2 * dp);
  float* nu = cv.take<float>(packed_norm_floats(pu.npad));
  if ((st = pack_points(ctx, A + k + (long long)c0 * lda, (int)lda, DB200_POINT_MAJOR, cols, w, dp, pu.npad, xu, nu)))
    return st;
  // column ranges of A22 (slices of the packed U12 sharing its scale), so that a trailing matrix of few 256-row
  // blocks still fills the 74 CTA pairs
  const int itiles = pl.npad / 256;
  int ranges = std::min((148 + itiles - 1) / itiles, (cols + 127) / 128);
  const int width = round_up((cols + ranges - 1) / ranges, 128);
  ranges = (cols + width - 1) / width;
  std::vector<TileJob> jobs((size_t)ranges);
  for (int q = 0; q < ranges; ++q) {
    const int j0 = q * width, nc = std::min(width, cols - j0);
    PackedPoints ps;
    ps.xp = static_cast<const uint16_t*>(xu) + (size_t)j0 * 2 * dp;
    ps.norms = nu + j0;
    ps.n = nc;
    ps.npad = round_up(nc, 128);  // within the parent's rows: j0 + npad <= roundup(cols, 128) <= pu.npad
    ps.dp = dp;
    ps.tail = nu + pu.npad;
    TileJob& J = jobs[(size_t)q];
    J.pi = pl;
    J.pj = ps;
    J.gamma = -1.0f;  // alpha: A22 -= L21 U12
    J.out = A + r0 + (long long)(c0 + j0) * lda;
    J.ldo = lda;
  }
  TilePlan T;
  if ((st = prepare_rbf_tiles(ctx, RBF_MODE_UPDATE, jobs.data(), ranges, nullptr, 0, &T))) return st;
  return launch_rbf_plan(ctx, T);
}

}  // namespace

int lu_factorize(db200_context* ctx, int m, int n, int nleft, float* A, long long lda, int* ipiv, int pivot,
                 int swap_left_panels) {
  const int mn = m < n ? m : n;
  int* singular = nullptr;
  // cooperative panel: scratch for the candidates, row j and the barrier counter; how many CTAs fit at once
  static_assert(CP_MAX_ROWS * W * 4 <= 200 * 1024, "panel slice too large");
  const size_t cp_smem = (size_t)CP_MAX_ROWS * W * sizeof(float);
  char* scr = static_cast<char*>(slot_buffer(ctx, SLOT_LA, 256 + 2 * 4096 * CAND * sizeof(float) + 2 * W * 4 + 256));
  if (!scr) return DB200_ERR_NOMEM;
  singular = reinterpret_cast<int*>(scr);
  unsigned* bar = reinterpret_cast<unsigned*>(scr + 64);
  int* cstatus = reinterpret_cast<int*>(scr + 128);
  float* cand = reinterpret_cast<float*>(scr + 256);
  float* rowj = cand + 2 * 4096 * CAND;
  DB200_CUDA(ctx, cudaMemsetAsync(scr, 0, 256, ctx->stream));
  int coop_max = 0;
  {
    int coop = 0, per_sm = 0;
    DB200_CUDA(ctx, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ctx->device));
    DB200_CUDA(ctx, cudaFuncSetAttribute(lu_panel_coop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)cp_smem));
    DB200_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lu_panel_coop_kernel, CP_THREADS,
                                                                  cp_smem));
    if (coop && per_sm > 0) coop_max = std::min(ctx->num_sms * per_sm, 4096);
  }
  // the cluster panel: the largest cluster (16, else the portable 8) of CTAs with full slices that fits
  int cl_max = 0;
  {
    DB200_CUDA(ctx, cudaFuncSetAttribute(lu_panel_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)cp_smem));
    const bool wide = cudaFuncSetAttribute(lu_panel_cluster_kernel,
                                           cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess;
    cudaGetLastError();
    for (int size : {CL_MAX, 8}) {
      if (size > 8 && !wide) continue;
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = (unsigned)size;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3((unsigned)size);
      cfg.blockDim = dim3(CL_THREADS);
      cfg.dynamicSmemBytes = cp_smem;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int clusters = 0;
      const bool fits = cudaOccupancyMaxActiveClusters(&clusters, lu_panel_cluster_kernel, &cfg) == cudaSuccess &&
                        clusters >= 1;
      cudaGetLastError();
      if (fits) {
        cl_max = size;
        break;
      }
    }
  }
  // the tensor-core trailing update: workspace for the largest (first) trailing matrix, taken before the loop so
  // that no later step reallocates it
  constexpr long long TC_MIN_ENTRIES = 1 << 20;
  void* tc_ws = nullptr;
  if ((long long)(m - W) * (n - W) >= TC_MIN_ENTRIES) {
    tc_ws = workspace(ctx, lu_update_tc_bytes(m, n));
    if (!tc_ws) return DB200_ERR_NOMEM;
  }
  unsigned bar_base = 0;
  for (int k = 0; k < mn; k += W) {
    const int w = mn - k < W ? mn - k : W;
    const int rows = m - k;
    // CTAs of at least 64 rows each, at most one slice of CP_MAX_ROWS per CTA
    int G = std::min(coop_max, (rows + 63) / 64);
    const int R = G > 0 ? (rows + G - 1) / G : 0;
    // cluster panel: up to cl_max CTAs of at least 256 rows (at least 1024 beyond 8 CTAs)
    int Gc = std::min(8, std::max(1, (rows + 255) / 256));
    if (rows > 8 * 1024) Gc = std::min(cl_max, (rows + 1023) / 1024);
    const int Rc = (rows + Gc - 1) / Gc;
    if (cl_max > 0 && Gc <= cl_max && Rc <= CP_MAX_ROWS) {
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = (unsigned)Gc;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3((unsigned)Gc);
      cfg.blockDim = dim3(CL_THREADS);
      cfg.dynamicSmemBytes = (size_t)Rc * W * sizeof(float);
      cfg.stream = ctx->stream;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      DB200_CUDA(ctx, cudaLaunchKernelEx(&cfg, lu_panel_cluster_kernel, A, lda, m, k, w, Rc, ipiv, pivot, singular));
    } else if (G > 0 && R <= CP_MAX_ROWS) {
      if (bar_base > 0x40000000u) {  // keep the monotone barrier target far from wrapping
        DB200_CUDA(ctx, cudaMemsetAsync(bar, 0, sizeof(unsigned), ctx->stream));
        bar_base = 0;
      }
      void* args[] = {&A, &lda, &m, &k, (void*)&w, (void*)&R, &ipiv, &pivot, &singular, &bar, &bar_base, &cand,
                      &rowj, &cstatus};
      DB200_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)lu_panel_coop_kernel, dim3((unsigned)G),
                                                  dim3(CP_THREADS), args, (size_t)R * W * sizeof(float),
                                                  ctx->stream));
      bar_base += (unsigned)w * (unsigned)G;
    } else {
      lu_panel_kernel<<<1, PANEL_THREADS, 0, ctx->stream>>>(A, lda, m, k, w, ipiv, pivot, singular);
    }
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
        if (tc_ws && (long long)(m - (k + w)) * cols >= TC_MIN_ENTRIES) {
          count_launch(ctx, launches);
          launches = 0;
          const int s2 = lu_update_tc(ctx, A, lda, m, n, k, w, k + w, k + w, tc_ws);
          if (s2) return s2;
        } else {
          dim3 grid((unsigned)((cols + UT - 1) / UT), (unsigned)((m - (k + w) + UT - 1) / UT));
          lu_update_kernel<<<grid, 256, 0, ctx->stream>>>(A, lda, m, n, k, w, k + w, k + w);
          DB200_CUDA(ctx, cudaGetLastError());
          ++launches;
        }
      }
    }
    count_launch(ctx, launches);
  }
  int sing = 0, to = 0;
  DB200_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, scr, 256, cudaMemcpyDeviceToHost, ctx->stream));
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::memcpy(&sing, ctx->h_pinned, sizeof(int));
  std::memcpy(&to, reinterpret_cast<char*>(ctx->h_pinned) + 128, sizeof(int));
  if (to) return fail(ctx, DB200_ERR_TIMEOUT, "lu_factorize: a panel's grid barrier gave up");
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
