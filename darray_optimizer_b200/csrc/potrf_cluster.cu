// Cholesky of a small SPD matrix in one launch on a thread-block cluster: the r x r capacity matrices of the
// barrier's Newton steps and the l x l Grams of CholeskyQR2 and the Nystrom core (l <= 544).
//
// The blocked right-looking algorithm of include/lapack_like.h:10-57 (potrf of the diagonal block, trsm of its
// block row, syrk of the trailing matrix) in 32-column steps, on the nc CTAs of one cluster, which keep the whole
// upper triangle in their shared memory: CTA c owns the columns j = c (mod nc), stored packed (column j holds rows
// 0..j).  One step, over the columns [c0, c0 + kb):
//   1. every CTA gathers the kb x kb diagonal block from its owners (distributed shared memory) and factors it
//      itself.  The same inputs and the same instructions give every CTA the same R11 bit for bit, so the block
//      is never broadcast, and a failing pivot stops every CTA at the same step;
//   2. each CTA solves R11^T x = a for its own columns right of the block (rows c0..c0 + kb - 1 of R, final), and
//      keeps them contiguous in its slot of the block row (the block row is stored by owner);
//   3. cluster barrier; each CTA stores R11 into its own columns of the block, copies every other CTA's slot
//      (16-byte distributed-shared-memory loads, contiguous) into its copy of the whole block row R12, and subtracts
//      R12^T R12 from its own columns right of the block (16 x 8 tiles on the FP64 tensor cores);
//   4. cluster barrier: the next diagonal block is complete and the slices may be overwritten.
// This replaces the multi-kernel path's two launches per 64 columns (diagonal block with its row, then the
// trailing update) with one launch whose data stays in shared memory from the first load to the final store
// (which also zeroes the strictly lower triangle).  The elimination inside the diagonal block is the one of
// potrf_block_kernel: rows are eliminated unscaled and divided by the square roots of their pivots at the end.
#include <algorithm>
#include <mutex>

#include "internal.h"
#include "la64.h"
#include "ptx.cuh"

namespace db200 {

namespace {

constexpr int PC_THREADS = 512;
constexpr int PC_WARPS = PC_THREADS / 32;
constexpr int PC_NB = 32;            // columns per step
constexpr int PC_MAX_L = 544;        // largest order: a cluster of 16 CTAs holds the triangle and the block row
constexpr int PC_MAX_NC = 16;
constexpr int PC_SMEM_LIMIT = 232448;
constexpr int PC_PAD = 128;          // doubles after the block row
constexpr int PC_DLD = PC_NB + 1;    // leading dimension of the staged diagonal block
constexpr int PC_PULL = 4;           // 16-byte distributed-shared-memory loads per thread in flight
constexpr int PC_QMAX = 64;          // own columns per CTA right of the first block (16 lanes x 4)
constexpr int PC_TCOLS = 4;          // columns a warp solves at once in the block-row substitution

// First element of CTA c's t-th own column (j = c + nc t, rows 0..j) in its packed storage.
__host__ __device__ inline int pc_col_off(int c, int nc, int t) { return t * (c + 1) + nc * (t * (t - 1) / 2); }

// Own columns of CTA c (count, and the first one right of column r0).
__host__ __device__ inline int pc_ncols(int c, int nc, int l) { return c < l ? (l - c + nc - 1) / nc : 0; }
__host__ __device__ inline int pc_first_right(int c, int nc, int r0) { return r0 > c ? (r0 - c + nc - 1) / nc : 0; }

// D[16x8] += A[16x8] B[8x8] in FP64 on the tensor cores (fragments of m16n8k8, g = lane / 4, t = lane % 4:
// A a0..a3 = A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4]; B b0, b1 = B[t][g], B[t+4][g];
// D d0, d1 = D[g][2t + 0, 1], d2, d3 = D[g+8][2t + 0, 1])
__device__ __forceinline__ void pc_dmma(double* d, const double* a, const double* b) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Shared memory (doubles, the same layout in every CTA, so that a location has the same offset in each):
//   own columns [own_cap] | block row R12 by owner: nc slots [32][qcap] + pad | diagonal block [32][33] |
//   1 / R_ii [32] | pivot rows [2][32] | failure flag and the update's owner table.  Slot o holds the rows c0..c0+kb-1 of CTA o's own columns right of the block, in their order.
__global__ void __launch_bounds__(PC_THREADS, 1) potrf_cluster_kernel(double* __restrict__ A, int lda, int l,
                                                                      int own_cap, int qcap, int* status, int* bad) {
  extern __shared__ __align__(16) double sm[];
  const int nc = (int)cluster_nctarank(), c = (int)cluster_ctarank();
  const int slot = PC_NB * qcap;
  double* own = sm;
  double* P = sm + own_cap;
  double* D = P + nc * slot + PC_PAD;
  double* dinv = D + PC_NB * PC_DLD;
  double* rowbuf = dinv + PC_NB;
  int* fail = reinterpret_cast<int*>(rowbuf + 2 * PC_NB);
  int* otab = fail + 4;  // [16] first own column right of the block, [16] their count, [16] spare, [17] tile prefix
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ncols = pc_ncols(c, nc, l);
  if (*(volatile int*)status) return;  // an earlier factorisation on this status word failed (same in every CTA)

  // the upper triangle of the own columns
  for (int t = warp; t < ncols; t += PC_WARPS) {
    const int j = c + nc * t;
    const double* col = A + (long long)j * lda;
    double* dst = own + pc_col_off(c, nc, t);
    for (int i = lane; i <= j; i += 32) dst[i] = col[i];
  }
  cluster_sync_all();

  const uint32_t own_s = smem_u32(own), P_s = smem_u32(P);
  for (int c0 = 0; c0 < l; c0 += PC_NB) {
    const int kb = min(PC_NB, l - c0);
    const int r0 = c0 + kb;  // first column right of the block
    // 1. the diagonal block, D[i][q] = A[c0 + i][c0 + q] for i <= q (a warp reads one column from its owner; both
    //    of a thread's loads are issued before either is stored)
    {
      double v[PC_NB * PC_NB / PC_THREADS];
#pragma unroll
      for (int u = 0; u < PC_NB * PC_NB / PC_THREADS; ++u) {
        const int e = tid + u * PC_THREADS, q = e >> 5, i = e & 31;
        v[u] = 0.0;
        if (q < kb && i <= q) {
          const int j = c0 + q, o = j % nc;
          const int idx = pc_col_off(o, nc, j / nc) + c0 + i;
          v[u] = (o == c) ? own[idx] : ld_shared_remote_f64(mapa_shared(own_s + 8u * (uint32_t)idx, (uint32_t)o));
        }
      }
#pragma unroll
      for (int u = 0; u < PC_NB * PC_NB / PC_THREADS; ++u) {
        const int e = tid + u * PC_THREADS;
        D[(e & 31) * PC_DLD + (e >> 5)] = v[u];
      }
    }
    __syncthreads();
    if (warp == 0) {
      // lane q holds column q; step i eliminates row i (its pivot in lane i, taken by a shuffle) from the rows
      // m > i, reading the row's entries from a shared copy (two buffers: the write of step i + 1 cannot meet a read
      // of step i)
      double a[PC_NB];
#pragma unroll
      for (int i = 0; i < PC_NB; ++i) a[i] = D[i * PC_DLD + lane];
      bool ok = true;
      double dg = 1.0;  // this lane's pivot
#pragma unroll
      for (int i = 0; i < PC_NB; ++i) {
        if (i >= kb) break;
        double* rb = rowbuf + (i & 1) * PC_NB;
        rb[lane] = a[i];
        const double piv = __shfl_sync(0xffffffffu, a[i], i);
        if (!(piv > 0.0)) {  // the same value in every lane (and in every CTA): a uniform exit
          ok = false;
          break;
        }
        if (lane == i) dg = piv;
        const double cq = a[i] * (1.0 / piv);
        __syncwarp();
#pragma unroll
        for (int m = i + 1; m < PC_NB; ++m)
          if (m <= lane) a[m] = fma(-rb[m], cq, a[m]);
      }
      __syncwarp();  // every lane is done with the row copies before they are reused
      if (ok) {
        // R[i][q] = U[i][q] / sqrt(U[i][i]) for the eliminated rows U
        const double rs = (lane < kb) ? 1.0 / sqrt(dg) : 0.0;
        rowbuf[lane] = rs;
        dinv[lane] = rs;
        __syncwarp();
#pragma unroll
        for (int i = 0; i < PC_NB; ++i) D[i * PC_DLD + lane] = (i <= lane && lane < kb) ? a[i] * rowbuf[i] : 0.0;
        if (lane < kb) D[lane * PC_DLD + lane] = sqrt(dg);
      }
      if (lane == 0) *fail = ok ? 0 : 1;
    }
    __syncthreads();
    if (*fail) {
      cluster_sync_all();  // no CTA leaves while another may still read its shared memory
      if (c == 0 && tid == 0 && atomicCAS(status, 0, DB200_ERR_NOT_SPD) == 0) *bad = c0;
      return;
    }
    // 2. rows c0..r0-1 of the own columns right of the block: R11^T x = a by forward substitution, a warp per 4
    //    columns (lane i holds row i of each; the 4 chains interleave), into the own column and the own slot
    const int t0 = pc_first_right(c, nc, r0);
    const int nown = ncols > t0 ? ncols - t0 : 0;
    for (int k0 = warp * PC_TCOLS; k0 < nown; k0 += PC_WARPS * PC_TCOLS) {
      const int nq = min(PC_TCOLS, nown - k0);
      double x[PC_TCOLS];
#pragma unroll
      for (int q = 0; q < PC_TCOLS; ++q)
        x[q] = (q < nq && lane < kb) ? own[pc_col_off(c, nc, t0 + k0 + q) + c0 + lane] : 0.0;
#pragma unroll
      for (int i = 0; i < PC_NB; ++i) {
        if (i >= kb) break;
        const double di = dinv[i], rij = D[i * PC_DLD + lane];  // R[i][lane] (0 for lanes at or above kb)
#pragma unroll
        for (int q = 0; q < PC_TCOLS; ++q) {
          const double xi = __shfl_sync(0xffffffffu, x[q], i) * di;
          if (lane == i) x[q] = xi;
          else if (lane > i) x[q] = fma(-rij, xi, x[q]);
        }
      }
      if (lane < kb) {
#pragma unroll
        for (int q = 0; q < PC_TCOLS; ++q) {
          if (q < nq) {
            own[pc_col_off(c, nc, t0 + k0 + q) + c0 + lane] = x[q];
            P[c * slot + lane * qcap + k0 + q] = x[q];
          }
        }
      }
    }
    cluster_sync_all();  // every slot is complete; every CTA has read its diagonal block
    // 3. R11 into the own columns of the block (no CTA gathers the block any more) ...
    for (int e = tid; e < kb * PC_NB; e += PC_THREADS) {
      const int q = e >> 5, i = e & 31;
      const int j = c0 + q;
      if (j % nc == c && i <= q) own[pc_col_off(c, nc, j / nc) + c0 + i] = D[i * PC_DLD + q];
    }
    //    ... the owner table of the update (first own column right of the block, their count, prefix of tiles) ...
    if (tid < nc) {
      const int t0o = pc_first_right(tid, nc, r0);
      otab[tid] = t0o;
      otab[PC_MAX_NC + tid] = pc_ncols(tid, nc, l) - t0o;
    }
    if (tid == 0) {
      const int ncb = (nown + 7) >> 3;
      int acc = 0;
      for (int o = 0; o < nc; ++o) {
        otab[3 * PC_MAX_NC + o] = acc;
        acc += ((pc_ncols(o, nc, l) - pc_first_right(o, nc, r0) + 15) >> 4) * ncb;
      }
      otab[3 * PC_MAX_NC + nc] = acc;
    }
    //    ... the other CTAs' slots, copied whole (kb rows of qcap) by 16-byte distributed-shared-memory loads,
    //    PC_PULL per thread in flight before their stores ...
    {
      // element e of the copy: source (c + 1 + oi) mod nc, offset 2 rem in its slot (row m, column pair ch:
      // m * qcap + 2 ch = 2 (m * qcap / 2 + ch)); a thread's e advances by PC_THREADS, so (oi, rem) are stepped
      const int per = kb * (qcap >> 1), total = (nc - 1) * per;
      int oi = tid / per, rem = tid - (tid / per) * per;
      for (int e0 = tid; e0 < total; e0 += PC_THREADS * PC_PULL) {
        double2 v[PC_PULL];
        int dst[PC_PULL];
#pragma unroll
        for (int u = 0; u < PC_PULL; ++u) {
          dst[u] = -1;
          if (e0 + u * PC_THREADS < total) {
            int src = c + 1 + oi;
            if (src >= nc) src -= nc;
            dst[u] = src * slot + 2 * rem;
            v[u] = ld_shared_remote_v2f64(mapa_shared(P_s + 8u * (uint32_t)dst[u], (uint32_t)src));
          }
          rem += PC_THREADS;
          if (rem >= per) {
            const int q = rem / per;
            oi += q;
            rem -= q * per;
          }
        }
#pragma unroll
        for (int u = 0; u < PC_PULL; ++u)
          if (dst[u] >= 0) *reinterpret_cast<double2*>(P + dst[u]) = v[u];
      }
    }
    __syncthreads();
    //    ... and the trailing update of the own columns right of the block on the FP64 tensor cores:
    //    A[i][j] -= sum_m R[m][i] R[m][j] for r0 <= i <= j.  A warp tile is 16 columns of one owner's slot (as rows
    //    i) x 8 own columns (as columns j), K = the block's kb rows in steps of 8 (mma.sync.m16n8k8.f64; fragments
    //    read straight from the slots, rows m >= kb read as zero).  Tiles wholly below the diagonal are skipped.
    {
      const int ncb = (nown + 7) >> 3;
      const int total = otab[3 * PC_MAX_NC + nc];  // tiles of all owners
      const int g8 = lane >> 2, t4 = lane & 3;
      const double* Pc = P + c * slot;
      int o = 0;  // the owner of tile it: walked forward as it grows
      for (int it = warp; it < total; it += PC_WARPS) {
        while (it >= otab[3 * PC_MAX_NC + o + 1]) ++o;
        const int t0o = otab[o], nso = otab[PC_MAX_NC + o];
        const int rest = it - otab[3 * PC_MAX_NC + o];
        const int rb = rest / ncb, cb = rest - rb * ncb;
        const int kq0 = 16 * rb, nb0 = 8 * cb;
        const int i_min = o + nc * (t0o + kq0);
        const int j_max = c + nc * (t0 + min(nown, nb0 + 8) - 1);
        if (i_min > j_max) continue;  // the whole tile lies below the diagonal (the same for every lane)
        const double* Po = P + o * slot + kq0;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int k0 = 0; k0 < PC_NB; k0 += 8) {
          if (k0 >= kb) break;
          const int ka = k0 + t4, kc = ka + 4;
          const bool va = ka < kb, vc = kc < kb;
          double af[4], bf[2];
          af[0] = va ? Po[ka * qcap + g8] : 0.0;
          af[1] = va ? Po[ka * qcap + g8 + 8] : 0.0;
          af[2] = vc ? Po[kc * qcap + g8] : 0.0;
          af[3] = vc ? Po[kc * qcap + g8 + 8] : 0.0;
          bf[0] = va ? Pc[ka * qcap + nb0 + g8] : 0.0;
          bf[1] = vc ? Pc[kc * qcap + nb0 + g8] : 0.0;
          pc_dmma(acc, af, bf);
        }
        // acc[0..1]: row kq0 + g8, own slot columns nb0 + 2 t4 + {0, 1}; acc[2..3]: row kq0 + g8 + 8
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int kq = kq0 + g8 + 8 * (e >> 1), nn = nb0 + 2 * t4 + (e & 1);
          if (kq >= nso || nn >= nown) continue;
          const int i = o + nc * (t0o + kq), j = c + nc * (t0 + nn);
          if (i <= j) own[pc_col_off(c, nc, t0 + nn) + i] -= acc[e];
        }
      }
    }
    cluster_sync_all();
  }

  // the factor, with the strictly lower triangle zeroed
  for (int t = warp; t < ncols; t += PC_WARPS) {
    const int j = c + nc * t;
    double* col = A + (long long)j * lda;
    const double* src = own + pc_col_off(c, nc, t);
    for (int i = lane; i < l; i += 32) col[i] = (i <= j) ? src[i] : 0.0;
  }
}

struct PcLayout {
  int own_cap, qcap;
  size_t bytes;
};

PcLayout pc_layout(int l, int nc) {
  PcLayout L;
  int own = 0, q = 0;
  for (int c = 0; c < nc && c < l; ++c) {
    own = std::max(own, pc_col_off(c, nc, pc_ncols(c, nc, l)));
    q = std::max(q, pc_ncols(c, nc, l) - pc_first_right(c, nc, std::min(l, PC_NB)));
  }
  L.own_cap = (own + 1) & ~1;  // the block row after it starts 16-byte aligned
  L.qcap = std::max(4, (q + 3) & ~3);  // a multiple of 4: a lane's 4 slot columns stay inside its row
  L.bytes = sizeof(double) * ((size_t)L.own_cap + (size_t)nc * PC_NB * L.qcap + PC_PAD + PC_NB * PC_DLD + 3 * PC_NB + 2 + 40);
  return L;
}

// Largest cluster the device can hold with PC_SMEM_LIMIT bytes per CTA (0: none), probed once per device.
int pc_nc_max(int device) {
  static std::mutex mu;
  static int cached[64];
  static bool done[64] = {};
  if (device < 0 || device >= 64) return 0;
  std::lock_guard<std::mutex> lock(mu);
  if (done[device]) return cached[device];
  int best = 0;
  if (cudaFuncSetAttribute(potrf_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, PC_SMEM_LIMIT) ==
      cudaSuccess) {
    const bool wide =
        cudaFuncSetAttribute(potrf_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess;
    for (int nc = wide ? PC_MAX_NC : 8; nc >= 1 && !best; --nc) {
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = (unsigned)nc;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3((unsigned)nc);
      cfg.blockDim = dim3(PC_THREADS);
      cfg.dynamicSmemBytes = PC_SMEM_LIMIT;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int clusters = 0;
      if (cudaOccupancyMaxActiveClusters(&clusters, potrf_cluster_kernel, &cfg) == cudaSuccess && clusters >= 1)
        best = nc;
    }
  }
  cudaGetLastError();
  cached[device] = best;
  done[device] = true;
  return best;
}

}  // namespace

void potrf_cluster_init(db200_context* ctx) { ctx->potrf_nc_max = pc_nc_max(ctx->device); }

int potrf_cluster_size(const db200_context* ctx, int l) {
  if (l < 1 || l > PC_MAX_L || ctx->potrf_nc_max < 1) return 0;
  const int nblk = (l + PC_NB - 1) / PC_NB;
  // about two 32-column blocks per CTA, more CTAs while the layout does not fit
  for (int nc = std::min(std::max(1, (nblk + 1) / 2), ctx->potrf_nc_max); nc <= ctx->potrf_nc_max; ++nc) {
    const PcLayout L = pc_layout(l, nc);
    if (L.bytes <= (size_t)PC_SMEM_LIMIT && L.qcap <= PC_QMAX) return nc;
  }
  return 0;
}

int potrf_cluster(db200_context* ctx, double* A, int lda, int l, int* d_status, int* d_bad) {
  const int nc = potrf_cluster_size(ctx, l);
  if (nc < 1) return DB200_ERR_UNSUPPORTED;
  const PcLayout L = pc_layout(l, nc);
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)nc;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3((unsigned)nc);
  cfg.blockDim = dim3(PC_THREADS);
  cfg.dynamicSmemBytes = L.bytes;
  cfg.stream = ctx->stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  DB200_CUDA(ctx, cudaLaunchKernelEx(&cfg, potrf_cluster_kernel, A, lda, l, L.own_cap, L.qcap, d_status, d_bad));
  count_launch(ctx);
  return DB200_OK;
}

}  // namespace db200
