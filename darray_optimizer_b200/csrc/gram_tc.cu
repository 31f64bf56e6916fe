// Tensor-core weighted Gram for the Woodbury capacity matrix of the Newton step:
//     M += Z~^T Z~,   Z~ = diag(sqrt(w)) Z   (Z: n x r FP64 column major, w = D^-1 >= 0)
// computed exactly in integers on the int8 tensor cores (the Ozaki splitting scheme: Ozaki, Ogita, Oishi and Rump,
// "Error-free transformations of matrix multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59 (2012); Ootomo, Ozaki and Yokota, "DGEMM on integer matrix multiplication
// unit", IJHPCA 2024).
//
//  1. The rows are cut into chunks of 16384.  In every chunk c each column p of Z~ is scaled by 2^-e_cp, e_cp the
//     exponent just above the chunk's largest |entry| of that column, so that x = Z~[i, p] 2^-e_cp lies in (-1, 1).
//  2. x is cut into KS signed 7-bit digits by truncation, x = sum_s d_s 2^-7s + (remainder < 2^-7 KS), d_s in
//     [-127, 127] (the base-128 digits of floor(|x| 2^(7 KS)) with the sign of x), stored as KS int8 slices
//     [s][p][i] (i contiguous).  One pass reads a column chunk (128 KB) for its maximum and again, from L2, to
//     slice it.
//  3. M[p, q] = sum_c 2^(e_cp + e_cq) sum_{s,t} 2^-7(s+t) (D_s^T D_t)_c[p, q].  The products with s + t <= KS + 1
//     are kept (the rest lie below the truncation); all products of one group g = s + t share a scale, so each
//     group is a single s32 accumulator in TMEM fed by tcgen05.mma kind::i8 (exact integer sums:
//     KS * 16384 * 127^2 < 2^31).  A CTA's k range lies inside one chunk.
//  4. The epilogue folds the groups in FP64 (Horner in 2^-7), scales by 2^(e_cp + e_cq) and adds the 128 x 64 tile
//     into M with FP64 atomics (the n dimension is split across CTAs).
//
// The result differs from the exact Z~^T Z~ by the dropped groups and the truncation only, about 2e-8, 3e-10,
// 3e-12, 3e-14 of ||Z~_p|| ||Z~_q|| for KS = 5, 6, 7, 8 (measured), next to FP64 accumulation's ~1e-16 sqrt(n).  The
// kernels are instantiated for each KS; the barrier solver
// still refines each Newton step against the exact FP64 operator and falls back to the FP64 Gram if refinement
// stalls.
#include <cuda.h>
#include <cooperative_groups.h>
#include <cudaTypedefs.h>
#include <algorithm>
#include <mutex>

#include "internal.h"
#include "ptx.cuh"

namespace db200 {
namespace {

constexpr int KS_MAX = 8;                      // int8 digits per value at most (groups g = s + t in [2, KS + 1])
constexpr int TM = 128;                        // M tile: rows p of M
constexpr int TN = 64;                         // N tile: columns q of M
constexpr int KB = 64;                         // k bytes per stage: one 64-byte swizzled row per operand row
constexpr int ASL = TM * KB;                   // one A slice per stage, 8 KB
constexpr int BSL = TN * KB;                   // one B slice per stage, 4 KB
template <int KS>
constexpr int stage_bytes() { return KS * (ASL + BSL); }  // 96 KB at 8 digits
constexpr int NSTAGE = 2;
constexpr int CH = 16384;                      // rows per scaling chunk (and at most per CTA: exact s32 sums)
constexpr int MAX_CHUNKS = CH / KB;            // k chunks (64 rows) per scaling chunk
constexpr int TMEM_COLS = 512;                 // KS * TN columns of s32 groups (at most 512)
constexpr int THREADS = 192;                   // warp 0 TMA, warp 1 MMA, warps 2..5 epilogue
static_assert(KS_MAX * TN <= TMEM_COLS, "group accumulators exceed TMEM");
static_assert((long long)KS_MAX * MAX_CHUNKS * KB * 127 * 127 < (1LL << 31), "s32 group sums could overflow");
constexpr int SLICE_CTAS = 4;                  // CTAs (of 256 threads x 16 rows) per scaling chunk
static_assert(SLICE_CTAS * 256 * 16 == CH && CH / SLICE_CTAS == 256 * 16, "slice_kernel covers a chunk per cluster");

struct GramArgs {
  int r;                // valid rows / columns of M
  int nq;               // q tiles (64 wide); p tiles are 128 high and tile pairs keep tj >= 2 ti
  int kchunks;          // npad / 64
  int chunks_per_split;  // divides MAX_CHUNKS: a CTA's k range lies in one scaling chunk
  int rpad;
  const int* exps;       // e_cp at [c * rpad + p]
  double* M;
  int ldm;
  int* status;
};

// e with m < 2^e for m >= 0 (floor(log2 m) + 1 from the IEEE exponent field); 0 for m == 0.
__device__ __forceinline__ int exp_above(double m) {
  const unsigned long long bits = (unsigned long long)__double_as_longlong(m);
  const int biased = (int)((bits >> 52) & 0x7ff);
  return bits == 0 ? 0 : biased - 1022;
}

template <int KS>
__global__ void __launch_bounds__(THREADS, 1)
    gram_i8_kernel(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_b, GramArgs g) {
  constexpr int STAGE = stage_bytes<KS>();
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t s_op = smem_u32(smem);
  const uint32_t s_bar = smem_u32(smem + NSTAGE * STAGE);
  auto full = [&](int s) { return s_bar + 8u * s; };
  auto empty = [&](int s) { return s_bar + 8u * (NSTAGE + s); };
  const uint32_t done = s_bar + 8u * (2 * NSTAGE);
  const uint32_t drain = s_bar + 8u * (2 * NSTAGE + 1);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + NSTAGE * STAGE + 256);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + NSTAGE * STAGE + 264);

  // tile pair (p tile ti, q tile tj >= 2 ti: the upper triangle) and k range of this CTA
  int idx = blockIdx.x, ti = 0;
  while (idx >= g.nq - 2 * ti) {
    idx -= g.nq - 2 * ti;
    ++ti;
  }
  const int tj = 2 * ti + idx;
  const int k0 = blockIdx.y * g.chunks_per_split;
  const int k1 = min(g.kchunks, k0 + g.chunks_per_split);
  const int nk = k1 - k0;

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (threadIdx.x == 0) {
    *abort_flag = 0;
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(full(s), 1);
      mbar_init(empty(s), 1);
    }
    mbar_init(done, 1);
    mbar_init(drain, 1);
    fence_mbarrier_init();
  }
  if (warp == 1) {
    tmem_alloc(smem_u32(tmem_slot), TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (nk > 0) {
      if (lane == 0) {
        prefetch_tmap(&tm_a);
        prefetch_tmap(&tm_b);
      }
      int issued = 0;
      for (int k = 0; k < nk; ++k) {
        const int s = k % NSTAGE;
        if (!__all_sync(0xffffffffu, mbar_wait(empty(s), ((k / NSTAGE) & 1) ^ 1, abort_flag))) break;
        if (elect_one()) {
          mbar_arrive_expect_tx(full(s), STAGE);
          const uint32_t base = s_op + s * STAGE;
          const int x = (k0 + k) * KB;
          tma_load_3d(base, &tm_a, full(s), x, ti * TM, 0);             // KS slices x 128 rows x 64 bytes
          tma_load_3d(base + KS * ASL, &tm_b, full(s), x, tj * TN, 0);  // KS slices x 64 rows x 64 bytes
        }
        __syncwarp();
        ++issued;
      }
      if (*abort_flag && lane == 0) {
        // let the copies in flight land before the CTA exits (bounded waits)
        volatile int never = 0;
        for (int k = (issued > NSTAGE ? issued - NSTAGE : 0); k < issued; ++k)
          mbar_wait(full(k % NSTAGE), (k / NSTAGE) & 1, &never);
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    const uint32_t idesc = idesc_i8(TM, TN);
    for (int k = 0; k < nk; ++k) {
      const int s = k % NSTAGE;
      if (!__all_sync(0xffffffffu, mbar_wait(full(s), (k / NSTAGE) & 1, abort_flag))) break;
      tc_fence_after();
      if (elect_one()) {
        const uint32_t base = s_op + s * STAGE;
        const uint32_t first = (k > 0) ? 1u : 0u;
#pragma unroll
        for (int sa = 0; sa < KS; ++sa) {
#pragma unroll
          for (int tb = 0; tb < KS - sa; ++tb) {
#pragma unroll
            for (int kk = 0; kk < KB / 32; ++kk) {
              const uint64_t da = sdesc_k_sw64(base + sa * ASL + kk * 32);
              const uint64_t db = sdesc_k_sw64(base + KS * ASL + tb * BSL + kk * 32);
              // group sa + tb is opened by its sa == 0 product in the first k chunk
              umma_i8(tmem + (uint32_t)((sa + tb) * TN), da, db, idesc, (sa > 0 || kk > 0) ? 1u : first);
            }
          }
        }
        umma_commit(empty(s));
      }
      __syncwarp();
    }
    if (elect_one()) {
      umma_commit(done);
      umma_commit(drain);
      volatile int never = 0;
      mbar_wait(drain, 0, &never);
    }
    __syncwarp();
  } else {
    const int q = warp & 3;  // TMEM lane quadrant
    const bool ok = (nk > 0) && __all_sync(0xffffffffu, mbar_wait(done, 0, abort_flag));
    if (ok) {
      tc_fence_after();
      const int row = ti * TM + 32 * q + lane;
      const int* ex = g.exps + (size_t)(k0 / MAX_CHUNKS) * g.rpad;
      const int ep = ex[row];
      for (int c0 = 0; c0 < TN; c0 += 16) {
        double v[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) v[e] = 0.0;
#pragma unroll
        for (int gi = KS - 1; gi >= 0; --gi) {
          float raw[16];
          tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(gi * TN + c0), raw);
          tmem_wait_ld();
#pragma unroll
          for (int e = 0; e < 16; ++e) v[e] = v[e] * 0.0078125 + (double)__float_as_int(raw[e]);
        }
        if (row < g.r) {
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const int col = tj * TN + c0 + e;
            if (col < g.r && row <= col)
              atomicAdd(g.M + (long long)col * g.ldm + row, ldexp(v[e], ep + ex[col] - 14));
          }
        }
      }
    }
    __syncwarp();
  }
  __syncthreads();
  if (threadIdx.x == 0 && *abort_flag) atomicExch(g.status, DB200_ERR_TIMEOUT);
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, TMEM_COLS);
  }
}

// sw[i] = sqrt(w_i) (1 without weights), computed once per Gram.
__global__ void sqrt_weights_kernel(const double* __restrict__ w, int n, double* __restrict__ sw) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) sw[i] = w ? sqrt(w[i]) : 1.0;
}

// One cluster of SLICE_CTAS CTAs (256 threads, 4096 rows each) per (column p < rpad, chunk c of 16384 rows).
//  1. Each thread loads 8 coalesced pairs of rows (lanes read adjacent 16-byte pairs) and keeps them in registers.
//  2. The CTAs exchange their largest |sw_i Z[i, p]| through distributed shared memory, which gives e_cp.
//  3. Each thread turns its 16 values into KS digits and parks them in a shared [KS][4096] byte tile.
//  4. The CTA writes every slice row out with coalesced 16-byte stores (zero for padding rows and columns).
// VEC: Z and ldz allow 16-byte loads.
template <bool VEC, int KS>
__global__ void __cluster_dims__(1, SLICE_CTAS, 1) __launch_bounds__(256)
    slice_kernel(const double* __restrict__ Z, long long ldz, const double* __restrict__ sw, int n, int r, int npad,
                 int rpad, int* __restrict__ exps, int8_t* __restrict__ slices) {
  constexpr int ROWS = CH / SLICE_CTAS;  // 4096 rows per CTA
  constexpr int ROUNDS = ROWS / 512;     // 8 rounds of 2 rows per thread
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int p = blockIdx.x, c = blockIdx.y / SLICE_CTAS;
  const int base = c * CH + rank * ROWS;  // first row of this CTA
  const double* col = Z + (long long)p * ldz;
  __shared__ __align__(16) uint8_t stage[KS][ROWS];
  __shared__ double part[8];
  __shared__ double cta_max;
  double v[2 * ROUNDS];
#pragma unroll
  for (int q = 0; q < ROUNDS; ++q) {
    const int i = base + 512 * q + 2 * threadIdx.x;
    if (p < r && VEC && i + 2 <= n) {
      const double2 z = __ldg(reinterpret_cast<const double2*>(col + i));
      const double2 ww = __ldg(reinterpret_cast<const double2*>(sw + i));
      v[2 * q] = ww.x * z.x;
      v[2 * q + 1] = ww.y * z.y;
    } else {
      v[2 * q] = (p < r && i < n) ? sw[i] * col[i] : 0.0;
      v[2 * q + 1] = (p < r && i + 1 < n) ? sw[i + 1] * col[i + 1] : 0.0;
    }
  }
  double m = 0.0;
#pragma unroll
  for (int j = 0; j < 2 * ROUNDS; ++j) m = fmax(m, fabs(v[j]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (threadIdx.x % 32 == 0) part[threadIdx.x / 32] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 1; k < 8; ++k) m = fmax(m, part[k]);
    cta_max = m;
  }
  cluster.sync();
#pragma unroll
  for (int k = 0; k < SLICE_CTAS; ++k) m = fmax(m, *cluster.map_shared_rank(&cta_max, k));
  cluster.sync();  // every CTA has read the others' maxima before any of them exits
  const int e = exp_above(m);
  if (rank == 0 && threadIdx.x == 0) exps[(size_t)c * rpad + p] = e;
  if (base >= npad) return;
  // floor(|x| 2^(7 KS)) with x = v 2^-e in (-1, 1): an exact fixed-point value below 2^(7 KS); digit s + 1 of |x|
  // in base 128 is bits [7 (KS - 1 - s), +7), negated (two's complement byte) for x < 0
  const double scale = ldexp(1.0, 7 * KS - e);
#pragma unroll
  for (int q = 0; q < ROUNDS; ++q) {
    const unsigned long long u0 = (m > 0.0) ? __double2ull_rz(fabs(v[2 * q]) * scale) : 0ull;
    const unsigned long long u1 = (m > 0.0) ? __double2ull_rz(fabs(v[2 * q + 1]) * scale) : 0ull;
    const uint32_t n0 = v[2 * q] < 0.0 ? 0xffu : 0u, n1 = v[2 * q + 1] < 0.0 ? 0xffu : 0u;
#pragma unroll
    for (int s = 0; s < KS; ++s) {
      const int sh = 7 * (KS - 1 - s);
      const uint32_t d0 = (uint32_t)(u0 >> sh) & 127u, d1 = (uint32_t)(u1 >> sh) & 127u;
      const uint32_t b0 = ((d0 ^ n0) - n0) & 0xffu, b1 = ((d1 ^ n1) - n1) & 0xffu;
      *reinterpret_cast<uint16_t*>(&stage[s][512 * q + 2 * threadIdx.x]) = (uint16_t)(b0 | (b1 << 8));
    }
  }
  __syncthreads();
  const size_t slice_bytes = (size_t)rpad * npad;
#pragma unroll
  for (int s = 0; s < KS; ++s) {
    const int off = 16 * threadIdx.x;  // 256 threads x 16 bytes = one 4096-row slice row
    if (base + off >= npad) break;     // npad is a multiple of 64: a 16-byte store is wholly inside or outside
    *reinterpret_cast<uint4*>(slices + s * slice_bytes + (size_t)p * npad + base + off) =
        *reinterpret_cast<const uint4*>(&stage[s][off]);
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, []() {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 3-D map over the slices (x = i bytes, y = p, z = slice), box 64 bytes x box_rows x KS, 64-byte swizzle.
bool tmap_slices(CUtensorMap* tm, const void* base, uint64_t npad, uint64_t rpad, uint32_t box_rows, int ks) {
  auto enc = encode_fn();
  if (!enc) return false;
  cuuint64_t dims[3] = {npad, rpad, (cuuint64_t)ks};
  cuuint64_t strides[2] = {npad, npad * rpad};
  cuuint32_t box[3] = {(cuuint32_t)KB, box_rows, (cuuint32_t)ks};
  cuuint32_t estr[3] = {1, 1, 1};
  return enc(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

size_t gram_tc_scratch_bytes(int n, int r) {
  const size_t npad = (size_t)round_up(n, KB), rpad = (size_t)round_up(r, TM);
  const size_t nchunk = (npad + CH - 1) / CH;
  return align_up((size_t)KS_MAX * npad * rpad, 256) + align_up(nchunk * rpad * sizeof(int), 256) +
         align_up((size_t)n * sizeof(double), 256) + 512;
}

namespace {
template <int KS>
int gram_tc_run(db200_context* ctx, int n, int r, const double* Z, long long ldz, const double* w, double* M,
                int ldm, void* scratch) {
  constexpr int STAGE = stage_bytes<KS>();
  if (n <= 0 || r <= 0) return DB200_OK;
  const int npad = round_up(n, KB), rpad = round_up(r, TM);
  const int nchunk = (npad + CH - 1) / CH;
  Carve cv{static_cast<char*>(scratch)};
  int8_t* slices = cv.take<int8_t>((size_t)KS * npad * rpad);
  int* exps = cv.take<int>((size_t)nchunk * rpad);
  double* sw = cv.take<double>(n);
  sqrt_weights_kernel<<<(unsigned)std::min((n + 255) / 256, 1024), 256, 0, ctx->stream>>>(w, n, sw);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  const bool vec = (reinterpret_cast<uintptr_t>(Z) % 16 == 0) && (ldz % 2 == 0);
  if (vec)
    slice_kernel<true, KS><<<dim3(rpad, nchunk * SLICE_CTAS), 256, 0, ctx->stream>>>(Z, ldz, sw, n, r, npad, rpad, exps,
                                                                                slices);
  else
    slice_kernel<false, KS><<<dim3(rpad, nchunk * SLICE_CTAS), 256, 0, ctx->stream>>>(Z, ldz, sw, n, r, npad, rpad, exps,
                                                                                 slices);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  CUtensorMap ta, tb;
  if (!tmap_slices(&ta, slices, npad, rpad, TM, KS) || !tmap_slices(&tb, slices, npad, rpad, TN, KS))
    return fail(ctx, DB200_ERR_CUDA, "gram_tc: cuTensorMapEncodeTiled failed");
  GramArgs a;
  a.r = r;
  a.rpad = rpad;
  a.exps = exps;
  const int np = rpad / TM;
  a.nq = round_up(r, TN) / TN;
  a.kchunks = npad / KB;
  const int pairs = np * a.nq - np * (np - 1);
  // k range per CTA: a power of two of 64-row chunks dividing the scaling chunk; pick the one with the least
  // modelled time, waves x (chunks per CTA + 8), the 8 standing for a CTA's fill and epilogue
  {
    const int sms = ctx->num_sms;
    long long best = -1;
    int best_cps = MAX_CHUNKS;
    for (int cps = MAX_CHUNKS; cps >= 4; cps /= 2) {
      const long long splits = (a.kchunks + cps - 1) / cps;
      const long long waves = (splits * pairs + sms - 1) / sms;
      const long long cost = waves * (long long)(cps + 8);
      if (best < 0 || cost < best) {
        best = cost;
        best_cps = cps;
      }
    }
    a.chunks_per_split = best_cps;
  }
  const int splits = (a.kchunks + a.chunks_per_split - 1) / a.chunks_per_split;
  if (splits > 65535) return fail(ctx, DB200_ERR_UNSUPPORTED, "gram_tc: too many row splits");
  a.M = M;
  a.ldm = ldm;
  a.status = ctx->d_status;
  const size_t smem = NSTAGE * STAGE + 512 + 1024;
  DB200_CUDA(ctx, cudaFuncSetAttribute(gram_i8_kernel<KS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(pairs, splits);
  cudaEvent_t e0 = nullptr;
  prof_begin(ctx, &e0);
  gram_i8_kernel<KS><<<grid, THREADS, smem, ctx->stream>>>(ta, tb, a);
  DB200_CUDA(ctx, cudaGetLastError());
  prof_end(ctx, e0);
  count_launch(ctx);
  return DB200_OK;
}
}  // namespace

// M (upper triangle, FP64, r x r) += Z~^T Z~ with Z~ = diag(sqrt(w)) Z from `slices` int8 digits per value (5..8;
// error about 2e-8, 3e-10, 3e-12, 3e-14 of ||Z~_p|| ||Z~_q||).  `scratch` holds gram_tc_scratch_bytes.
int gram_tc_weighted(db200_context* ctx, int n, int r, const double* Z, long long ldz, const double* w, double* M,
                     int ldm, void* scratch, int slices) {
  switch (slices) {
    case 5: return gram_tc_run<5>(ctx, n, r, Z, ldz, w, M, ldm, scratch);
    case 6: return gram_tc_run<6>(ctx, n, r, Z, ldz, w, M, ldm, scratch);
    case 7: return gram_tc_run<7>(ctx, n, r, Z, ldz, w, M, ldm, scratch);
    case 8: return gram_tc_run<8>(ctx, n, r, Z, ldz, w, M, ldm, scratch);
    default: return fail(ctx, DB200_ERR_INVALID, "gram_tc: slices must be 5..8");
  }
}

}  // namespace db200
