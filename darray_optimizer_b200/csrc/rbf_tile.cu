// Fused RBF-kernel tile engine for sm_100a (tcgen05 + TMEM + TMA).
//
// Squared distances use the GEMM form ||x||^2 + ||y||^2 - 2 x.y of include/dkernel.cu:116-129.  Each point set is
// scaled by one power of two 2^e (largest |coordinate| just below 2^14, so every product and sum stays far inside
// fp16 and fp32) and split into fp16 hi + lo (22 significant bits; a bf16 split keeps 16, whose representation
// error ~2^-17 |x| left the dual objective 3e-6 from FP64 at n = 4096, d = 32).  The norms are formed from the
// same split products as the cross term, so the sum cancels to fp32 round-off on the diagonal instead of leaving
// the split's representation error.  The epilogue undoes the scales: x.y = 2^-(e_I + e_J) G.
//
// A CTA pair (cluster of 2) owns a 256-row block of points i and one panel of sketch columns.  It streams every
// 128-column block of points j and, per tile:
//   MMA1  G   = Xi . Xj^T  in TMEM (fp32), from split-fp16 operands: hi.hi + hi.lo + lo.hi
//   epi   P   = exp2(min(a_i + b_j + c G, 0)),  a = -gamma*log2(e)*||x||^2,  c = 2*gamma*log2(e) 2^-(e_I+e_J)
//   MMA2  Y  += P . Omega~_j   (SKETCH mode; P is written to tensor memory as the fp16 A operand, Omega~ is fp16)
//         or  K[i, j] = y_i y_j P   stored as fp32 (KBLOCK mode)
//         or  out[i, j] += alpha 2^-(e_I+e_J) G, no exp (UPDATE mode: the split-fp16 product of a rank-d update, e.g.
//             the trailing update of a blocked LU, with x_i the rows of L21 and x_j the columns of U12)
//         or  the 8 smallest d_ij^2 = |x_i|^2 + |x_j|^2 - 2 x.y of each row per column quarter, kept sorted in registers
//             across the j tiles (KNN mode: k-nearest-neighbour distances; a second kernel merges the quarters)
// so the kernel matrix is never written to HBM in SKETCH mode.  Algorithm restated from
// include/dkernel.cu:102-129 (vecnorm, rbf) and :151-178 / :194-231 (distance GEMM, rbf, sketch GEMM).
//
// Compensated sketch (SKETCH mode, per instance): P is also split into fp16 hi + lo (P_lo = fp16(P - P_hi), in a
// second 64-column TMEM tile) and Omega~ into hi + lo rows, and MMA2 issues P_hi.Om_hi + P_lo.Om_hi (+ P_hi.Om_lo)
// into the same fp32 accumulator: ~22-bit operands instead of 11.  The single fp16 product's rounding of P (2^-12
// of a kernel value, which at n = 131072 is half the size of the sketch's tail entries) moves the range finder's
// subspace enough to leave the dual objective ~4e-4 from FP64; the compensated product brings it to ~1e-7.
//
// Both MMAs are issued by the pair leader as tcgen05 cta_group::2 instructions with M = 256: each CTA supplies its
// own 128 rows of A (Xi in shared memory, P in tensor memory) and half of the rows of B (Xj, Omega~), and holds
// the accumulators (G, Y) of its own rows.  Per CTA, warp roles (608 threads): warp 0 = TMA producer of the point
// tiles, warp 18 = TMA producer of the sketch operand, warp 1 = TMEM allocator (both CTAs) + MMA issuer (leader),
// warps 2..17 = epilogue (four warps per TMEM lane quadrant, each owning 32 of the 128 tile columns).  Sixteen
// epilogue warps keep the exp/pack of one tile shorter than the distance MMA of the next, so the P tile is ready
// when the tensor pipe reaches it; P is handed over in two halves (j 0..63, 64..127), one per K chunk of the
// sketch MMA.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

#include "internal.h"
#include "ptx.cuh"

namespace db200 {

namespace {

constexpr int BM = 128;                    // rows of i per CTA (TMEM lanes)
constexpr int PAIR_M = 256;                // rows of i per CTA pair (UMMA M of the 2-SM instructions)
constexpr int BN = 128;                    // columns of j per tile
constexpr int BN_HALF = BN / 2;            // rows of Xj each CTA of the pair holds per tile
constexpr int KC = 64;                     // 16-bit elements per 128-byte swizzled row chunk
constexpr int XI_CHUNK = BM * KC * 2;      // 128 x 64 fp16 = 16 KB
constexpr int XJ_CHUNK = BN_HALF * KC * 2; // 64 x 64 fp16 = 8 KB
constexpr int NUM_EPI_WARPS = 16;
constexpr int EPI_COLS = BN / (NUM_EPI_WARPS / 4);  // tile columns per epilogue warp (32)
constexpr int OM_WARP = 2 + NUM_EPI_WARPS;          // Omega producer warp (18)
constexpr int NUM_THREADS = 32 * (OM_WARP + 1);     // 608
constexpr int TMEM_COLS = 512;
constexpr int SMEM_LIMIT = 232448;  // dynamic shared memory per block on sm_100
constexpr int BAR_BYTES = 1024;     // barrier region: barriers, TMEM slot, abort flag
constexpr int MAX_NSX = 16, MAX_NSO = 4;
constexpr float LOG2E = 1.4426950408889634f;

// One instance of the tile engine.  A launch walks a work list over a table of instances in global memory (one
// instance for the single-problem entry points, many for the batched one); work item k belongs to the instance
// with the largest item_begin <= k and covers one 256-row block of its points i and one panel of its sketch.
struct alignas(64) TileInst {
  CUtensorMap tm_xi, tm_xj, tm_om1, tm_om2;  // packed points (rows i, rows j) and the two Omega~ row boxes
  const float* si;       // squared norms, padded to n_itiles * 256 / n_jtiles * 128
  const float* sj;
  const float* fi;       // the point sets' scales 2^-e of the packed operands (one float each)
  const float* fj;
  const unsigned* lof_i;  // nonzero when some point of the set has a nonzero lo part (written by the pack)
  const unsigned* lof_j;
  const float* yi;
  const float* yj;
  float* out;
  long long ldo;
  int m, n;              // valid rows / columns
  int n_itiles, n_jtiles, n_panels, panel, l;  // n_itiles counts 256-row pair tiles
  int n1, n2;            // sketch MMA split of the panel: N = n1 (+ n2) columns, n2 = 0 for one instruction
  int g_bufs;            // 1 or 2 TMEM buffers of 128 columns for G
  int tmem_p, tmem_y;    // first TMEM column of the P tile (64 columns, 128 with P_lo) and of the Y panel
  int nkc;               // 64-element chunks per packed row [hi | lo]: 1..4 (feature pad 32..128)
  int comp;              // sketch product: 0 = P.Om, 1 = + P_lo.Om, 2 = + P_hi.Om_lo (compensated)
  int om_lo;             // row offset of the Omega~ lo rows inside the packed operand (comp = 2)
  int promote;           // j tiles per TMEM accumulation chunk, each chunk added into Y in fp32 (0: whole item)
  int item_begin;        // first work item of this instance
  float c_row, c_dot;    // -gamma*log2e, 2*gamma*log2e
};

struct LaunchArgs {
  // A one-instance launch carries its tensor maps as kernel parameters (read through the constant bank);
  // batched launches read them from the instance table in global memory.
  CUtensorMap tm1[4];
  const TileInst* inst;
  int count, n_items;
  int nsx, nso;          // Xj and Omega ring stages
  int nkc_max, panel_max;  // shared-memory layout covers every instance
  int om_mult;           // Omega stage copies: 1, or 2 when an instance loads hi and lo rows (comp = 2)
  int* status;
};

struct SmemLayout {
  int om_stage;  // bytes of one Omega stage in one CTA: (panel / 2) rows x 128 B, twice with lo rows
  size_t off_xi, off_xj, off_om, off_sj, off_bar, total;
};
constexpr int SJ_BYTES = NUM_EPI_WARPS * 2 * EPI_COLS * 4;  // per epilogue warp: two tiles' column norms

__host__ __device__ inline SmemLayout make_layout(int nkc, int panel, int nsx, int nso, int om_mult) {
  SmemLayout L;
  L.om_stage = (panel / 2) * 128 * om_mult;
  L.off_xi = 0;
  L.off_xj = L.off_xi + (size_t)nkc * XI_CHUNK;
  L.off_om = L.off_xj + (size_t)nsx * XJ_CHUNK;
  L.off_sj = L.off_om + (size_t)nso * L.om_stage;
  L.off_bar = L.off_sj + SJ_BYTES;
  L.total = L.off_bar + BAR_BYTES;
  return L;
}

// Barrier slots (8 bytes each) after off_bar.  "leader" barriers are only used in CTA 0 of the pair (the MMA
// issuer waits on them; CTA 1 arrives remotely or its TMA completes on them); "pair" barriers exist in both CTAs
// and are signalled by the leader's multicast tcgen05.commit.
enum {
  B_XI_FULL = 0,  // leader: both CTAs' Xi bytes
  B_XI_EMPTY,     // pair
  B_G_FULL0,      // pair
  B_G_FULL1,
  B_G_EMPTY0,     // leader: 2 x NUM_EPI_WARPS arrivals
  B_G_EMPTY1,
  B_P_FULL0,      // leader: P half h, 2 x NUM_EPI_WARPS / 2 arrivals
  B_P_FULL1,
  B_P_EMPTY0,     // pair
  B_P_EMPTY1,
  B_Y_FULL,       // pair
  B_Y_EMPTY,      // leader: 2 x NUM_EPI_WARPS arrivals
  B_DRAIN,        // pair
  B_XJ_FULL0,     // nsx full (leader), nsx empty (pair), nso full (leader), nso empty (pair)
};
constexpr int TMEM_SLOT_OFF = 960, ABORT_OFF = 968;
static_assert((B_XJ_FULL0 + 2 * MAX_NSX + 2 * MAX_NSO) * 8 <= TMEM_SLOT_OFF, "barrier region too small");

// work item k -> instance (binary search over item_begin; the table is tiny and cached)
__device__ __forceinline__ int find_inst(const TileInst* inst, int count, int k) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&inst[mid].item_begin) <= k) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int V>
using IntC = std::integral_constant<int, V>;

// State of the MMA issuer: ring positions and phases, carried across tiles, items and instances.
struct Issuer {
  uint32_t tmem_base, s_bar, om_stage16;
  uint64_t dxi, dxj, dom;
  int nsx, nso, XJ_FULL, XJ_EMPTY, OM_FULL, OM_EMPTY;
  volatile int* abort_flag;
  uint32_t xs, xph, os, oph, pph;
  uint32_t guse0, guse1, gnext;  // uses of G buffer 0 / 1 (their phases) and the next buffer to fill
  uint32_t ydone;                // Y accumulations committed to the epilogue so far (B_Y_FULL phases)
};

__device__ __forceinline__ bool issuer_wait(const Issuer& S, int idx, uint32_t parity) {
  return __all_sync(0xffffffffu, mbar_wait(S.s_bar + 8u * (uint32_t)idx, parity, S.abort_flag));
}

// Distance MMA of one tile into the next G buffer, for a packed row of 2 * DP elements (split fp16).  EXACT: both
// point sets are exact in fp16 after scaling (every lo is zero, e.g. 0/1 features), so only hi.hi is issued; the
// lo chunks still pass through the Xj ring.
template <int DP, bool EXACT>
__device__ __forceinline__ bool issue_mma1(Issuer& S, int g_bufs) {
  constexpr uint32_t idesc_g = idesc_f16(PAIR_M, BN, false);
  constexpr int NKC = (2 * DP) / KC;
  const uint32_t gbuf = S.gnext;
  const uint32_t guse = gbuf ? S.guse1 : S.guse0;
  if (!issuer_wait(S, B_G_EMPTY0 + (int)gbuf, (guse & 1) ^ 1)) return false;
  tc_fence_after();
  const uint32_t d_tmem = S.tmem_base + gbuf * BN;
#pragma unroll
  for (int c = 0; c < NKC; ++c) {
    if (!issuer_wait(S, S.XJ_FULL + (int)S.xs, S.xph)) return false;
    tc_fence_after();
    if (elect_one()) {
      const uint64_t bbase = S.dxj + ((S.xs * XJ_CHUNK) >> 4);
#pragma unroll
      for (int ks = 0; ks < KC / 16; ++ks) {
        const int o = c * KC + ks * 16;  // K offset of this slice inside the packed row [hi | lo]
        const uint64_t bdesc = bbase + ((ks * 32) >> 4);
        if (o < DP) {  // B slice is hi_j: pair with hi_i and lo_i
          const int oh = o, ol = DP + o;
          umma_f16_pair(d_tmem, S.dxi + (((oh / KC) * XI_CHUNK + (oh % KC) * 2) >> 4), bdesc, idesc_g,
                        o == 0 ? 0u : 1u);
          if (!EXACT)
            umma_f16_pair(d_tmem, S.dxi + (((ol / KC) * XI_CHUNK + (ol % KC) * 2) >> 4), bdesc, idesc_g, 1u);
        } else if (!EXACT) {  // B slice is lo_j: pair with hi_i
          const int oh = o - DP;
          umma_f16_pair(d_tmem, S.dxi + (((oh / KC) * XI_CHUNK + (oh % KC) * 2) >> 4), bdesc, idesc_g, 1u);
        }
      }
      umma_commit_pair(S.s_bar + 8u * (uint32_t)(S.XJ_EMPTY + (int)S.xs));
      if (c == NKC - 1) umma_commit_pair(S.s_bar + 8u * (uint32_t)(B_G_FULL0 + (int)gbuf));
    }
    __syncwarp();
    if (++S.xs == (uint32_t)S.nsx) { S.xs = 0; S.xph ^= 1; }
  }
  if (gbuf) ++S.guse1;
  else ++S.guse0;
  S.gnext = (g_bufs == 2) ? (gbuf ^ 1u) : 0u;
  return true;
}

// Per-item constants of the sketch MMA.
struct SketchMma {
  uint32_t idesc_y1, idesc_y2, y2_boff, lo_boff, tmem_p, tmem_y, tmem_y2;
};

// Sketch MMA of one tile: two K chunks of 64, one per P half.  fp16 operands (P in [0, 1], Omega~ Gaussian: both
// well inside fp16 range, 3 more mantissa bits than bf16 at the same tensor rate).  COMP >= 1 adds P_lo.Om_hi
// (P_lo 64 TMEM columns after P_hi), COMP = 2 also P_hi.Om_lo (the lo rows follow the hi rows in each Omega
// stage); compensated panels take one instruction (N <= 256).
template <bool TWO, int COMP>
__device__ __forceinline__ bool issue_mma2(Issuer& S, const SketchMma& Y, int jt) {
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    // K chunk c of the sketch MMA reads P half c (j in [64c, 64c + 64))
    if (!issuer_wait(S, B_P_FULL0 + c, S.pph)) return false;
    if (!issuer_wait(S, S.OM_FULL + (int)S.os, S.oph)) return false;
    tc_fence_after();
    if (elect_one()) {
      const uint64_t bbase = S.dom + S.os * S.om_stage16;
#pragma unroll
      for (int ks = 0; ks < KC / 16; ++ks) {
        // A = P (fp16 in TMEM, 8 columns per 16-wide K step), B = Omega~ rows of this panel
        const uint32_t a_tmem = Y.tmem_p + c * 32 + ks * 8;
        const uint64_t bdesc = bbase + ((ks * 32) >> 4);
        const uint32_t acc = (jt > 0 || c > 0 || ks > 0) ? 1u : 0u;
        umma_f16_ts_pair(Y.tmem_y, a_tmem, bdesc, Y.idesc_y1, acc);
        if (TWO) umma_f16_ts_pair(Y.tmem_y2, a_tmem, bdesc + Y.y2_boff, Y.idesc_y2, acc);
        if (COMP >= 1) umma_f16_ts_pair(Y.tmem_y, a_tmem + 64, bdesc, Y.idesc_y1, 1u);
        if (COMP >= 2) umma_f16_ts_pair(Y.tmem_y, a_tmem, bdesc + Y.lo_boff, Y.idesc_y1, 1u);
      }
      umma_commit_pair(S.s_bar + 8u * (uint32_t)(S.OM_EMPTY + (int)S.os));
      umma_commit_pair(S.s_bar + 8u * (uint32_t)(B_P_EMPTY0 + c));
    }
    __syncwarp();
    if (++S.os == (uint32_t)S.nso) { S.os = 0; S.oph ^= 1; }
  }
  S.pph ^= 1;
  return true;
}

// All MMAs of one work item (every j tile, distance MMA one tile ahead of the sketch MMA), specialised for the
// instance's feature width and panel split so the hot loop carries no dispatch.  With promote = T > 0 the sketch
// accumulator restarts every T tiles: each chunk is committed to the epilogue, which adds it into Y in fp32
// (round to nearest), and the next chunk waits for that drain.  The tensor cores' fp32 accumulation truncates, so
// a sum over all n points loses ~2^-25 of its value per accumulation step, always toward zero; chunks of T tiles
// bound that loss by the steps in one chunk.
template <int MODE, int DP, bool TWO, int COMP, bool EXACT>
__device__ __forceinline__ bool issue_item(Issuer& S, const SketchMma& Y, int njt, int g_bufs, int promote) {
  if (!issue_mma1<DP, EXACT>(S, g_bufs)) return false;
  for (int jt = 0; jt < njt; ++jt) {
    if (jt + 1 < njt && !issue_mma1<DP, EXACT>(S, g_bufs)) return false;
    if (MODE == RBF_MODE_SKETCH) {
      const int jc = promote ? jt % promote : jt;  // tile inside the accumulation chunk (0: fresh accumulator)
      if (promote && jc == 0 && jt > 0) {
        if (!issuer_wait(S, B_Y_EMPTY, (S.ydone - 1) & 1)) return false;
        tc_fence_after();
      }
      if (!issue_mma2<TWO, COMP>(S, Y, jc)) return false;
      if (promote && (jc == promote - 1 || jt == njt - 1)) {
        if (elect_one()) umma_commit_pair(S.s_bar + 8u * (uint32_t)B_Y_FULL);
        __syncwarp();
        ++S.ydone;
      }
    }
  }
  return true;
}

template <int MODE, bool TWO, int COMP, bool EXACT>
__device__ __forceinline__ bool issue_item_dpx(Issuer& S, const SketchMma& Y, int nkc, int njt, int g_bufs,
                                               int promote) {
  switch (nkc) {
    case 1: return issue_item<MODE, 32, TWO, COMP, EXACT>(S, Y, njt, g_bufs, promote);
    case 2: return issue_item<MODE, 64, TWO, COMP, EXACT>(S, Y, njt, g_bufs, promote);
    case 3: return issue_item<MODE, 96, TWO, COMP, EXACT>(S, Y, njt, g_bufs, promote);
    default: return issue_item<MODE, 128, TWO, COMP, EXACT>(S, Y, njt, g_bufs, promote);
  }
}

template <int MODE, bool TWO, int COMP>
__device__ __forceinline__ bool issue_item_dp(Issuer& S, const SketchMma& Y, int nkc, int njt, int g_bufs,
                                              int promote, bool exact) {
  return exact ? issue_item_dpx<MODE, TWO, COMP, true>(S, Y, nkc, njt, g_bufs, promote)
               : issue_item_dpx<MODE, TWO, COMP, false>(S, Y, nkc, njt, g_bufs, promote);
}

// Dispatch of one work item to the loop specialised for its panel split and sketch product (KBLOCK items and
// compensated panels take one instruction).
template <int MODE>
__device__ __forceinline__ bool issue_item_any(Issuer& S, const SketchMma& Y, int nkc, int njt, int g_bufs, bool two,
                                               int comp, int promote, bool exact) {
  if (MODE != RBF_MODE_SKETCH) return issue_item_dpx<MODE, false, 0, false>(S, Y, nkc, njt, g_bufs, 0);
  if (comp == 2) return issue_item_dp<MODE, false, 2>(S, Y, nkc, njt, g_bufs, promote, exact);
  if (comp == 1) return issue_item_dp<MODE, false, 1>(S, Y, nkc, njt, g_bufs, promote, exact);
  return two ? issue_item_dp<MODE, true, 0>(S, Y, nkc, njt, g_bufs, promote, exact)
             : issue_item_dp<MODE, false, 0>(S, Y, nkc, njt, g_bufs, promote, exact);
}

// fp32 add into global memory performed in L2 without returning the old value (red, not atom: the warp does not
// wait for a reply)
__device__ __forceinline__ void red_add_f32(float* p, float v) {
  asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

// Drain of the sketch accumulator by one epilogue warp: its 32 rows (TMEM lanes from t_lane) x panel/4 columns,
// 8 columns per TMEM load batch.  accumulate: add into Y with fp32 reductions (red.global.add, round to nearest,
// performed in L2) instead of storing.  A reduction does not wait for the old value, so the drain costs no global
// load latency (a load-add-store drain made the pass 2x slower).  Every element has one owner thread, whose first
// chunk stores and later chunks add, in program order to the same address.  Kept out of line: its registers
// would otherwise stay reserved across the epilogue's exp loop.
__device__ __noinline__ void drain_sketch_chunk(const TileInst* I, int item, uint32_t rank, int row, int qc,
                                                uint32_t t_lane_base, bool accumulate) {
  const int li = item - I->item_begin;
  const int pn = li / I->n_itiles, m = I->m;
  const int i = (li % I->n_itiles) * PAIR_M + (int)rank * BM + row;
  float* const out_i = I->out + i;
  const long long ldo = I->ldo;
  const float y_i = (i < m && I->yi) ? I->yi[i] : 1.0f;
  const int panel = I->panel, l = I->l;
  const int quarter = panel / 4;  // panel is a multiple of 16
  for (int cc = 0; cc < quarter; cc += 8) {
    float yv[8];
    const int nc = min(8, quarter - cc);  // 4 or 8
    const uint32_t ta = t_lane_base + I->tmem_y + qc * quarter + cc;
    tmem_ld4(ta, yv);
    if (nc > 4) tmem_ld4(ta + 4, yv + 4);
    tmem_wait_ld();
    if (i < m) {
      const int col0 = pn * panel + qc * quarter + cc;
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        if (e < nc && col0 + e < l) {
          float* dst = out_i + (size_t)(col0 + e) * ldo;
          if (accumulate) red_add_f32(dst, y_i * yv[e]);
          else *dst = y_i * yv[e];
        }
      }
    }
  }
}

// One CTA pair (cluster of 2) owns a 256-row block of points i (128 rows per CTA, rank r holds rows 128r..) and one
// panel of sketch columns.  The leader (rank 0) issues every MMA as cta_group::2 with M = 256: A (Xi, P) is each
// CTA's own 128 rows, B (Xj, Omega~) is split by rows between the two CTAs, the accumulators (G, Y) sit in each
// CTA's tensor memory for its own rows.  Each CTA loads its own operand halves with TMA and the completion is
// counted on the leader's barrier.  All rings and barrier phases run on across work items and instances.
// LEAN (SKETCH launches whose every instance takes the single product without promotion): the compensated
// product's residual split and the promoted accumulation's chunk drains are compiled out of the epilogue, whose
// arithmetic sits on the critical path of the single-product pass (2.5 ms of 33 ms at C2 in the general form).
template <int MODE, bool LEAN>
__global__ void __launch_bounds__(NUM_THREADS, 1) rbf_tile_kernel(const __grid_constant__ LaunchArgs args) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const SmemLayout L = make_layout(args.nkc_max, args.panel_max, args.nsx, args.nso, args.om_mult);
  const int nsx = args.nsx, nso = args.nso;
  const uint32_t s_xi = smem_u32(smem + L.off_xi);
  const uint32_t s_xj = smem_u32(smem + L.off_xj);
  const uint32_t s_om = smem_u32(smem + L.off_om);
  const uint32_t s_bar = smem_u32(smem + L.off_bar);
  auto bar = [&](int idx) -> uint32_t { return s_bar + 8u * (uint32_t)idx; };
  const int XJ_FULL = B_XJ_FULL0, XJ_EMPTY = B_XJ_FULL0 + nsx, OM_FULL = XJ_EMPTY + nsx, OM_EMPTY = OM_FULL + nso;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + L.off_bar + TMEM_SLOT_OFF);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L.off_bar + ABORT_OFF);

  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  const uint32_t rank = cluster_ctarank();
  const bool leader = (rank == 0);
  const int cid = (int)cluster_id_x(), ncl = (int)cluster_count_x();
  const int n_items = args.n_items;
  // leader-side barrier addresses in the shared::cluster window
  auto lbar = [&](int idx) -> uint32_t { return mapa_shared(bar(idx), 0); };
  // a wait that gives up also stops the other CTA of the pair
  auto give_up = [&]() { st_shared_remote_u32(mapa_shared(smem_u32((const void*)abort_flag), rank ^ 1u), 1u); };

  if (threadIdx.x == 0) {
    *abort_flag = 0;
    mbar_init(bar(B_XI_FULL), 1);
    mbar_init(bar(B_XI_EMPTY), 1);
    mbar_init(bar(B_G_FULL0), 1);
    mbar_init(bar(B_G_FULL1), 1);
    mbar_init(bar(B_G_EMPTY0), 2 * NUM_EPI_WARPS);
    mbar_init(bar(B_G_EMPTY1), 2 * NUM_EPI_WARPS);
    mbar_init(bar(B_P_FULL0), NUM_EPI_WARPS);
    mbar_init(bar(B_P_FULL1), NUM_EPI_WARPS);
    mbar_init(bar(B_P_EMPTY0), 1);
    mbar_init(bar(B_P_EMPTY1), 1);
    mbar_init(bar(B_Y_FULL), 1);
    mbar_init(bar(B_Y_EMPTY), 2 * NUM_EPI_WARPS);
    mbar_init(bar(B_DRAIN), 1);
    for (int s = 0; s < nsx; ++s) {
      mbar_init(bar(XJ_FULL + s), 1);
      mbar_init(bar(XJ_EMPTY + s), 1);
    }
    for (int s = 0; s < nso; ++s) {
      mbar_init(bar(OM_FULL + s), 1);
      mbar_init(bar(OM_EMPTY + s), 1);
    }
    fence_mbarrier_init();
  }
  if (warp == 1) {
    tmem_alloc_pair(smem_u32(tmem_slot), TMEM_COLS);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  cluster_sync_all();  // barriers initialised and TMEM allocated in both CTAs before any cross-CTA traffic
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0 || warp == OM_WARP) {
    // ------------------------------------------------------------ TMA producers (both CTAs)
    if (lane == 0) {
      const bool points = (warp == 0);
      uint32_t xs = 0, xph = 0, os = 0, oph = 0, items_done = 0;
      int last = -1;
      bool ok = true;
      for (int item = cid; item < n_items && ok; item += ncl, ++items_done) {
        const int b = find_inst(args.inst, args.count, item);
        const TileInst* I = args.inst + b;
        const int li = item - I->item_begin;
        const int it = li % I->n_itiles, pn = li / I->n_itiles;
        const int nkc = I->nkc, njt = I->n_jtiles;
        const bool one = (args.count == 1);
        const CUtensorMap* t_xi = one ? &args.tm1[0] : &I->tm_xi;
        const CUtensorMap* t_xj = one ? &args.tm1[1] : &I->tm_xj;
        const CUtensorMap* t_om1 = one ? &args.tm1[2] : &I->tm_om1;
        const CUtensorMap* t_om2 = one ? &args.tm1[3] : &I->tm_om2;
        if (b != last) {
          if (points) {
            prefetch_tmap(t_xi);
            prefetch_tmap(t_xj);
          } else if (MODE == RBF_MODE_SKETCH) {
            prefetch_tmap(t_om1);
            if (I->n2 > 0) prefetch_tmap(t_om2);
          }
          last = b;
        }
        if (points) {
          if (!mbar_wait(bar(B_XI_EMPTY), (items_done & 1) ^ 1, abort_flag)) { ok = false; break; }
          if (leader) mbar_arrive_expect_tx(bar(B_XI_FULL), 2 * nkc * XI_CHUNK);
          for (int c = 0; c < nkc; ++c)
            tma_load_2d_pair(s_xi + c * XI_CHUNK, t_xi, lbar(B_XI_FULL), c * KC, it * PAIR_M + (int)rank * BM);
        }
        const int n1 = I->n1, n2 = I->n2, panel = I->panel;
        const int om_lo = (I->comp == 2) ? I->om_lo : -1;  // lo rows of Omega~ follow the hi rows in each stage
        for (int jt = 0; jt < njt && ok; ++jt) {
          if (points) {
            for (int c = 0; c < nkc; ++c) {
              if (!mbar_wait(bar(XJ_EMPTY + xs), xph ^ 1, abort_flag)) { ok = false; break; }
              if (leader) mbar_arrive_expect_tx(bar(XJ_FULL + xs), 2 * XJ_CHUNK);
              tma_load_2d_pair(s_xj + xs * XJ_CHUNK, t_xj, lbar(XJ_FULL + xs), c * KC,
                               jt * BN + (int)rank * BN_HALF);
              if (++xs == (uint32_t)nsx) { xs = 0; xph ^= 1; }
            }
          } else if (MODE == RBF_MODE_SKETCH) {
            for (int c = 0; c < 2; ++c) {
              if (!mbar_wait(bar(OM_EMPTY + os), oph ^ 1, abort_flag)) { ok = false; break; }
              if (leader) mbar_arrive_expect_tx(bar(OM_FULL + os), panel * 128 * (om_lo >= 0 ? 2 : 1));
              // rows of this CTA: [r*n1/2, (r+1)*n1/2) of the first instruction's n1 columns, then the same
              // half of the second instruction's n2 columns (or, compensated, of the lo rows)
              const uint32_t dst = s_om + os * L.om_stage;
              const int x = jt * BN + c * KC, y0 = pn * panel;
              tma_load_2d_pair(dst, t_om1, lbar(OM_FULL + os), x, y0 + (int)rank * (n1 / 2));
              if (n2 > 0)
                tma_load_2d_pair(dst + (n1 / 2) * 128, t_om2, lbar(OM_FULL + os), x,
                                 y0 + n1 + (int)rank * (n2 / 2));
              if (om_lo >= 0)
                tma_load_2d_pair(dst + (n1 / 2) * 128, t_om1, lbar(OM_FULL + os), x,
                                 om_lo + y0 + (int)rank * (n1 / 2));
              if (++os == (uint32_t)nso) { os = 0; oph ^= 1; }
            }
          }
        }
      }
      if (!ok) {
        give_up();
        // Loads this lane issued complete on the leader's barriers, which this CTA cannot observe: give them
        // time to land in shared memory before the pair tears down (bulk copies take microseconds).
        const uint64_t t0 = global_timer_ns();
        while (global_timer_ns() - t0 < 200000ull) {
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer (leader CTA only)
    // The whole warp runs the schedule converged and waits together; one elected lane issues each block of
    // MMAs.  Within a block every branch is resolved at compile time: the feature width and the panel split are
    // dispatched once per work item to specialised loops, since a lone issuing lane that waits on mbarriers or
    // branches between MMAs cannot keep the tensor pipe fed.
    if (leader) {
      Issuer S;
      S.tmem_base = tmem_base;
      S.s_bar = s_bar;
      S.om_stage16 = (uint32_t)L.om_stage >> 4;
      // Descriptors are affine in the shared address (start address in the low 14 bits, in 16-byte units):
      // build the base descriptors once and add offsets.
      S.dxi = sdesc_k_sw128(s_xi);
      S.dxj = sdesc_k_sw128(s_xj);
      S.dom = sdesc_k_sw128(s_om);
      S.nsx = nsx;
      S.nso = nso;
      S.XJ_FULL = XJ_FULL;
      S.XJ_EMPTY = XJ_EMPTY;
      S.OM_FULL = OM_FULL;
      S.OM_EMPTY = OM_EMPTY;
      S.abort_flag = abort_flag;
      S.xs = S.xph = S.os = S.oph = S.pph = 0;
      S.guse0 = S.guse1 = 0;
      S.gnext = 0;
      S.ydone = 0;
      uint32_t items_done = 0;
      bool ok = true;
      for (int item = cid; item < n_items && ok; item += ncl, ++items_done) {
        // every per-instance value in registers before the tile loop (no global reads between MMAs)
        const TileInst* I = args.inst + find_inst(args.inst, args.count, item);
        const int nkc = I->nkc, njt = I->n_jtiles, g_bufs = I->g_bufs;
        const int n1 = I->n1, n2 = I->n2;
        const bool two = n2 > 0;
        SketchMma Y;
        Y.idesc_y1 = idesc_f16(PAIR_M, n1, false);
        Y.idesc_y2 = idesc_f16(PAIR_M, two ? n2 : 16, false);
        Y.y2_boff = (uint32_t)((n1 / 2) * 128) >> 4;
        Y.lo_boff = Y.y2_boff;  // compensated panels take one instruction: the lo rows sit where n2's would
        const int comp = LEAN ? 0 : I->comp, promote = LEAN ? 0 : I->promote;
        // both point sets exact in fp16 after scaling (no lo part anywhere): hi.hi only
        const bool exact = (MODE == RBF_MODE_SKETCH) && (*I->lof_i | *I->lof_j) == 0u;
        Y.tmem_p = tmem_base + (uint32_t)I->tmem_p;
        Y.tmem_y = tmem_base + (uint32_t)I->tmem_y;
        Y.tmem_y2 = Y.tmem_y + (uint32_t)n1;
        if (!issuer_wait(S, B_XI_FULL, items_done & 1)) { ok = false; break; }
        tc_fence_after();
        if (MODE == RBF_MODE_SKETCH && S.ydone > 0) {
          // the previous item's Y (and P) columns may overlap this instance's G buffers: wait for the drain
          if (!issuer_wait(S, B_Y_EMPTY, (S.ydone - 1) & 1)) { ok = false; break; }
          tc_fence_after();
        }
        ok = issue_item_any<MODE>(S, Y, nkc, njt, g_bufs, two, comp, promote, exact);
        if (!ok) break;
        if (elect_one()) {
          umma_commit_pair(bar(B_XI_EMPTY));
          if (MODE == RBF_MODE_SKETCH && !promote) umma_commit_pair(bar(B_Y_FULL));
        }
        __syncwarp();
        if (MODE == RBF_MODE_SKETCH && !promote) ++S.ydone;
      }
      if (!ok && lane == 0) give_up();
      // All MMAs issued by this warp must be complete before TMEM is released (in both CTAs).
      if (elect_one()) umma_commit_pair(bar(B_DRAIN));
      __syncwarp();
    }
    volatile int never = 0;
    mbar_wait(bar(B_DRAIN), 0, &never);
    __syncwarp();
  } else if (warp >= 2 && warp < 2 + NUM_EPI_WARPS) {
    // ------------------------------------------------------------ epilogue (both CTAs, own rows)
    const int ew = warp - 2;              // 0..15
    const int q = warp & 3;               // TMEM lane quadrant this warp may access
    const int qc = ew >> 2;               // column quarter of the tile (32 columns)
    const int h = qc >> 1;                // P half (K chunk of the sketch MMA) these columns belong to
    const int row = 32 * q + lane;        // row inside this CTA's 128 rows
    const uint32_t t_lane = (uint32_t)(32 * q) << 16;
    // Column norms of this warp's 32 columns, double-buffered per warp in shared memory: lane l fetches the value
    // for the next tile from global memory before the current tile's exp, and parks it here afterwards, so the
    // global latency never sits between a G tile and its P tile.
    float* sjbuf = reinterpret_cast<float*>(smem + L.off_sj) + ew * 2 * EPI_COLS;
    uint32_t kp = 0, items_done = 0, ydone = 0;  // ydone: Y accumulations drained (B_Y_FULL phases)
    uint32_t guse0 = 0, guse1 = 0, gnext = 0;  // the same G-buffer sequence as the MMA issuer
    bool ok = true;
    for (int item = cid; item < n_items && ok; item += ncl, ++items_done) {
      const TileInst* I = args.inst + find_inst(args.inst, args.count, item);
      const int li = item - I->item_begin;
      const int it = li % I->n_itiles, pn = li / I->n_itiles;
      const int njt = I->n_jtiles, g_bufs = I->g_bufs, m = I->m;
      const bool p_lo = !LEAN && (I->comp >= 1);
      const int promote = (MODE == RBF_MODE_SKETCH && !LEAN) ? I->promote : 0;
      const float c_row = I->c_row;
      const float* sj = I->sj;
      const uint32_t t_p = tmem_base + t_lane + (uint32_t)I->tmem_p + (uint32_t)(qc * (EPI_COLS / 2));
      const long long ldo = I->ldo;
      const int n_cols = I->n;
      const float* const yj_all = I->yj;
      const int i = it * PAIR_M + (int)rank * BM + row;
      float* const out_i = I->out + i;
      const float a_i = c_row * I->si[i];  // si is padded to n_itiles * PAIR_M
      const float c_dot = I->c_dot * *I->fi * *I->fj;  // x_i.x_j = 2^-(e_I + e_J) G
      const float y_i = (i < m && I->yi) ? I->yi[i] : 1.0f;
      sjbuf[lane] = sj[qc * EPI_COLS + lane];  // tile 0 of this item
      __syncwarp();
      float best[8];  // KNN: this row's 8 smallest squared distances in this column quarter, ascending
#pragma unroll
      for (int t = 0; t < 8; ++t) best[t] = INFINITY;
      bool pending_drain = false, pending_acc = false;
      auto drain = [&](bool accumulate) -> bool {
        if (!__all_sync(0xffffffffu, mbar_wait(bar(B_Y_FULL), ydone & 1, abort_flag))) return false;
        tc_fence_after();
        drain_sketch_chunk(I, item, rank, row, qc, tmem_base + t_lane, accumulate);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_remote(lbar(B_Y_EMPTY));
        ++ydone;
        return true;
      };
      for (int jt = 0; jt < njt; ++jt) {
        // sj is padded to n_jtiles * BN
        const float sj_next = (jt + 1 < njt) ? sj[(jt + 1) * BN + qc * EPI_COLS + lane] : 0.0f;
        const uint32_t b = gnext;
        const uint32_t guse = b ? guse1 : guse0;
        if (!__all_sync(0xffffffffu, mbar_wait(bar(B_G_FULL0 + b), guse & 1, abort_flag))) { ok = false; break; }
        tc_fence_after();
        if (b) ++guse1;
        else ++guse0;
        gnext = (g_bufs == 2) ? (b ^ 1u) : 0u;
        float v[EPI_COLS];
        const uint32_t tcol = tmem_base + t_lane + b * BN + qc * EPI_COLS;
        tmem_ld16(tcol, v);
        tmem_ld16(tcol + 16, v + 16);
        tmem_wait_ld();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_remote(lbar(B_G_EMPTY0 + b));

        const int j0 = jt * BN + qc * EPI_COLS;
        if (MODE == RBF_MODE_KNN) {
          // d^2 = |x_i|^2 + |x_j|^2 - 2 x.y (x.y = c_dot G), inserted into the sorted list; padding columns and the
          // point itself skipped
          const float* sjt = sjbuf + (jt & 1) * EPI_COLS;
          const int* idx_j = reinterpret_cast<const int*>(yj_all);
          const float s_i = I->si[i];
#pragma unroll
          for (int c = 0; c < EPI_COLS; ++c) {
            const int j = j0 + c;
            const float d2 = fmaf(-2.0f * c_dot, v[c], s_i + sjt[c]);
            if (j < n_cols && d2 < best[7] && __ldg(idx_j + j) != i) {
              float x = d2;
#pragma unroll
              for (int t = 0; t < 8; ++t) {  // insertion: x moves down while it is smaller
                const float lo = fminf(best[t], x), hi = fmaxf(best[t], x);
                best[t] = lo;
                x = hi;
              }
            }
          }
        }
        if (MODE != RBF_MODE_UPDATE && MODE != RBF_MODE_KNN) {
          const float4* sj4 = reinterpret_cast<const float4*>(sjbuf + (jt & 1) * EPI_COLS);
#pragma unroll
          for (int c = 0; c < EPI_COLS / 4; ++c) {
            const float4 s4 = sj4[c];
            v[4 * c + 0] = fast_exp2(fminf(fmaf(c_dot, v[4 * c + 0], fmaf(c_row, s4.x, a_i)), 0.0f));
            v[4 * c + 1] = fast_exp2(fminf(fmaf(c_dot, v[4 * c + 1], fmaf(c_row, s4.y, a_i)), 0.0f));
            v[4 * c + 2] = fast_exp2(fminf(fmaf(c_dot, v[4 * c + 2], fmaf(c_row, s4.z, a_i)), 0.0f));
            v[4 * c + 3] = fast_exp2(fminf(fmaf(c_dot, v[4 * c + 3], fmaf(c_row, s4.w, a_i)), 0.0f));
          }
        }

        sjbuf[((jt + 1) & 1) * EPI_COLS + lane] = sj_next;
        __syncwarp();
        if (MODE == RBF_MODE_SKETCH) {
          // P_hi = fp16(P); with the compensated product also P_lo = fp16(P - P_hi), the exact residual of the hi
          // rounding (|P_lo| <= 2^-12 P), written 64 TMEM columns after P_hi
          uint32_t pk[EPI_COLS / 2], pl[EPI_COLS / 2];
#pragma unroll
          for (int c = 0; c < EPI_COLS / 2; ++c) {
            const __half2 hh = __floats2half2_rn(v[2 * c], v[2 * c + 1]);
            pk[c] = *reinterpret_cast<const uint32_t*>(&hh);
            if (!LEAN) {
              const float2 hf = __half22float2(hh);
              pl[c] = pack_f16x2(v[2 * c] - hf.x, v[2 * c + 1] - hf.y);
            }
          }
          if (!__all_sync(0xffffffffu, mbar_wait(bar(B_P_EMPTY0 + h), (kp & 1) ^ 1, abort_flag))) {
            ok = false;
            break;
          }
          tc_fence_after();
          // P row = this thread's row; j in [32qc, 32qc + 32) -> TMEM columns tmem_p + 16qc .. + 15
          tmem_st16(t_p, pk);
          if (p_lo) tmem_st16(t_p + 64, pl);
          tmem_wait_st();
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive_remote(lbar(B_P_FULL0 + h));
          ++kp;
          // A chunk closed by the previous tile is drained only now, after this tile's P is handed over: the
          // distance MMA of the next tile (whose G buffer this tile just read) then runs during the drain, and only
          // the sketch MMA of this tile waits for it.
          // Up to two drains here (one call site): the chunk closed by the previous tile, then, on the item's last
          // tile, the chunk this tile closes (nothing follows it to overlap with).  The first chunk of an item
          // stores, later chunks add.
          const bool closes = promote && ((jt + 1) % promote == 0 || jt == njt - 1);
          bool dq[2] = {pending_drain, closes && jt == njt - 1};
          bool da[2] = {pending_acc, jt >= promote};
          pending_drain = closes && jt < njt - 1;
          pending_acc = jt >= promote;
          for (int dd = 0; dd < 2 && ok; ++dd)
            if (dq[dd] && !drain(da[dd])) ok = false;
          if (!ok) break;
        } else if (MODE == RBF_MODE_KNN) {
          // (the list was updated above)
        } else if (MODE == RBF_MODE_UPDATE) {
          // each (i, j) has one owner thread: a plain read-modify-write, 8 columns at a time with every load
          // issued before the first store (the stores could alias the loads, so interleaved they would serialise)
          if (i < m) {
#pragma unroll
            for (int hh = 0; hh < EPI_COLS; hh += 8) {
              float o[8];
#pragma unroll
              for (int c = 0; c < 8; ++c) {
                const int j = j0 + hh + c;
                o[c] = (j < n_cols) ? out_i[(size_t)j * ldo] : 0.0f;
              }
#pragma unroll
              for (int c = 0; c < 8; ++c) {
                const int j = j0 + hh + c;
                if (j < n_cols) out_i[(size_t)j * ldo] = fmaf(c_dot, v[hh + c], o[c]);
              }
            }
          }
        } else {
          if (i < m) {
#pragma unroll
            for (int c = 0; c < EPI_COLS; ++c) {
              const int j = j0 + c;
              if (j < n_cols) {
                const float yj = yj_all ? __ldg(yj_all + j) : 1.0f;
                out_i[(size_t)j * ldo] = y_i * yj * v[c];
              }
            }
          }
        }
      }
      if (!ok) break;
      if (MODE == RBF_MODE_KNN && i < m) {
        float* o = I->out + (size_t)i * 32 + qc * 8;
#pragma unroll
        for (int t = 0; t < 8; ++t) o[t] = best[t];
      }
      if (MODE == RBF_MODE_SKETCH && !promote) {
        if (!drain(false)) { ok = false; break; }
      }
    }
    if (!ok && lane == 0) give_up();
    __syncwarp();
  }

  // Neither CTA may leave (or free TMEM) while the other can still touch its shared memory or tensor memory:
  // every role above ends after a bounded wait, then the pair meets here.
  tc_fence_before();
  cluster_sync_all();
  tc_fence_after();
  if (threadIdx.x == 0 && *abort_flag) atomicExch(args.status, DB200_ERR_TIMEOUT);
  if (warp == 1) tmem_dealloc_pair(tmem_base, TMEM_COLS);
}

// ------------------------------------------------------------------ packing kernels
// Largest |x_ik| of a point set (non-negative floats order like their bit patterns): block maxima, then one
// atomicMax per block into *out, which the caller zeroes first.
__global__ void absmax_points_kernel(const float* __restrict__ X, long long sp, long long sf, int n, int d,
                                     unsigned* __restrict__ out) {
  const long long total = (long long)n * d;
  float mx = 0.f;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = e / d, k = e % d;
    const float a = fabsf(X[i * sp + k * sf]);
    if (a <= 3.0e38f) mx = fmaxf(mx, a);  // NaN and inf do not set the scale
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  __shared__ float wmax[32];
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x / 32] = mx;
  __syncthreads();
  if (threadIdx.x < 32) {
    mx = (threadIdx.x < blockDim.x / 32) ? wmax[threadIdx.x] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (threadIdx.x == 0) atomicMax(out, __float_as_uint(mx));
  }
}

// One warp per point.  Every point of the set is scaled by the same 2^e, e = 14 - ceil(log2 max |x_ik|) (largest
// |coordinate| in [2^13, 2^14)), and split into fp16 hi = fp16(2^e x), lo = fp16(2^e x - hi).  norms[i] =
// ||x||^2 (0 on padding rows) and norms[npad + 1] = 2^-e; norms[npad] holds the set's max |x| bits from
// absmax_points_kernel, and norms[npad + 2] becomes nonzero when some lo part is (zeroed beforehand).  d <= dp <= 128, so each lane holds its (up to 4) coordinates in registers.
__global__ void pack_points_kernel(const float* __restrict__ X, long long sp, long long sf, int n, int d, int dp,
                                   int npad, __half* __restrict__ Xp, float* __restrict__ norms) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x / 32);
  const float mx = __uint_as_float(*reinterpret_cast<const unsigned*>(norms + npad));
  int e = 0;
  if (mx > 0.f) {
    int ex = 0;
    frexpf(mx, &ex);  // mx = f 2^ex, f in [0.5, 1)
    e = min(max(14 - ex, -120), 120);
  }
  const float sc = ldexpf(1.0f, e);
  if (blockIdx.x == 0 && threadIdx.x == 0) norms[npad + 1] = ldexpf(1.0f, -e);
  unsigned* lo_flag = reinterpret_cast<unsigned*>(norms + npad + 2);
  for (long long i = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; i < npad; i += warps) {
    float acc = 0.f;
    bool has_lo = false;
    __half* row = Xp + i * (2 * dp);
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int k = lane + 32 * t;
      if (k < dp) {
        const float x = ((i < n && k < d) ? X[i * sp + (long long)k * sf] : 0.f) * sc;  // exact: power of two
        const __half hi = __float2half_rn(x);
        const __half lo = __float2half_rn(x - __half2float(hi));
        row[k] = hi;
        row[dp + k] = lo;
        // ||x||^2 from the same split products the distance MMA forms (hi.hi + 2 hi.lo), so that
        // ||x||^2 + ||y||^2 - 2 x.y cancels to ~fp32 round-off for coincident points
        const float h = __half2float(hi), l = __half2float(lo);
        acc = fmaf(h, h, fmaf(2.0f * h, l, acc));
        if (l != 0.0f) has_lo = true;
      }
    }
    if (__any_sync(0xffffffffu, has_lo) && lane == 0) atomicOr(lo_flag, 1u);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) norms[i] = ldexpf(acc, -2 * e);
  }
}

// Omega~^T rows in fp16: Op[c][j] = fp16(y_j Omega[j + c*ldo]) for c < lrows; with `comp`, rows lrows + c hold
// the lo parts fp16(y_j Omega - hi).
__global__ void pack_sketch_kernel(const float* __restrict__ Om, long long ldo, const float* __restrict__ yj, int n,
                                   int l, int njpad, int lrows, int comp, __half* __restrict__ Op) {
  const long long total = (long long)njpad * lrows;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(e % njpad);
    const int c = (int)(e / njpad);
    float v = 0.f;
    if (j < n && c < l) v = Om[j + (long long)c * ldo] * (yj ? yj[j] : 1.0f);
    const __half hi = __float2half_rn(v);
    Op[e] = hi;
    if (comp) Op[total + e] = __float2half_rn(v - __half2float(hi));
  }
}

// ------------------------------------------------------------------ host helpers
PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, []() {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 2-D 16-bit tensor map: inner dimension `inner` (elements, contiguous), `outer` rows of pitch `pitch_elems`,
// box 64 x box_rows, 128-byte swizzle.
bool make_tmap(CUtensorMap* tm, const void* base, uint64_t inner, uint64_t outer, uint64_t pitch_elems,
               uint32_t box_rows, CUtensorMapDataType dtype = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16) {
  auto enc = get_encode();
  if (!enc) return false;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {pitch_elems * 2};
  cuuint32_t box[2] = {64, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(tm, dtype, 2, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

cudaLaunchConfig_t launch_config(cudaLaunchAttribute* attr, int clusters, size_t smem, cudaStream_t st) {
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(2 * clusters));
  cfg.blockDim = dim3(NUM_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

// Persistent grid size: as many CTA pairs as can be resident at once, no more than there are items.  Not
// stream-ordered (so launches can be captured in a CUDA graph afterwards).
template <int MODE, bool LEAN>
cudaError_t plan_clusters(size_t smem, int max_clusters, int n_items, int* clusters) {
  auto k = rbf_tile_kernel<MODE, LEAN>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = launch_config(attr, max_clusters, smem, nullptr);
  int resident = 0;
  e = cudaOccupancyMaxActiveClusters(&resident, k, &cfg);
  if (e != cudaSuccess) return e;
  if (resident < 1) return cudaErrorInvalidConfiguration;
  int c = resident < max_clusters ? resident : max_clusters;
  if (c > n_items) c = n_items;
  *clusters = c;
  return cudaSuccess;
}

template <int MODE, bool LEAN>
cudaError_t launch_kernel(const LaunchArgs& a, size_t smem, int clusters, cudaStream_t st) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = launch_config(attr, clusters, smem, st);
  return cudaLaunchKernelEx(&cfg, rbf_tile_kernel<MODE, LEAN>, a);
}

}  // namespace

int feature_pad(int d) { return round_up(d < 1 ? 1 : d, 32); }

// Sketch panels: with one 128-column G buffer, P (64 columns) and Y fit a panel of up to 320 columns; with two
// G buffers, up to 192.  Take whichever needs fewer panels (ties: two G buffers, which overlap better).  The
// compensated product (comp >= 1) keeps P_lo beside P (128 columns): panels of up to 256 / 128 columns.
SketchPlan plan_sketch(int l, int comp) {
  SketchPlan p;
  const int pcols = comp ? 128 : 64;
  const int w1 = TMEM_COLS - 128 - pcols, w2 = TMEM_COLS - 256 - pcols;
  const int lpad = round_up(l < 1 ? 1 : l, 16);
  const int np1 = (lpad + w1 - 1) / w1, np2 = (lpad + w2 - 1) / w2;
  p.g_bufs = (np2 <= np1) ? 2 : 1;
  p.n_panels = (p.g_bufs == 2) ? np2 : np1;
  p.panel = round_up((lpad + p.n_panels - 1) / p.n_panels, 16);
  p.lrows = p.n_panels * p.panel;
  p.comp = comp;
  return p;
}

int pack_points(db200_context* ctx, const float* X, int ldx, int layout, int n, int d, int dp, int npad, void* xp,
                float* norms) {
  const long long sp = (layout == DB200_POINT_MAJOR) ? ldx : 1;
  const long long sf = (layout == DB200_POINT_MAJOR) ? 1 : ldx;
  unsigned* mx = reinterpret_cast<unsigned*>(norms + npad);
  DB200_CUDA(ctx, cudaMemsetAsync(mx, 0, 4 * sizeof(unsigned), ctx->stream));  // max |x|, scale, lo flag
  if (n > 0) {
    long long mblocks = ((long long)n * d + 255) / 256;
    if (mblocks > (long long)ctx->num_sms * 4) mblocks = (long long)ctx->num_sms * 4;
    absmax_points_kernel<<<(unsigned)mblocks, 256, 0, ctx->stream>>>(X, sp, sf, n, d, mx);
    DB200_CUDA(ctx, cudaGetLastError());
    count_launch(ctx);
  }
  const int threads = 256;
  long long blocks = ((long long)npad * 32 + threads - 1) / threads;
  if (blocks > 65535LL * 4) blocks = 65535LL * 4;
  pack_points_kernel<<<(unsigned)blocks, threads, 0, ctx->stream>>>(X, sp, sf, n, d, dp, npad,
                                                                    static_cast<__half*>(xp), norms);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

int pack_sketch(db200_context* ctx, const float* Omega, int ldo, const float* yj, int n, int l, int njpad, int lrows,
                void* op, int comp) {
  const long long total = (long long)njpad * lrows;
  long long blocks = (total + 255) / 256;
  if (blocks > (long long)ctx->num_sms * 32) blocks = (long long)ctx->num_sms * 32;
  pack_sketch_kernel<<<(unsigned)blocks, 256, 0, ctx->stream>>>(Omega, ldo, yj, n, l, njpad, lrows,
                                                                comp == 2 ? 1 : 0, static_cast<__half*>(op));
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  return DB200_OK;
}

size_t tile_table_bytes(int count) { return (size_t)count * sizeof(TileInst); }

int prepare_rbf_tiles(db200_context* ctx, int mode, const TileJob* jobs, int count, void* table_storage,
                      size_t table_capacity, TilePlan* plan) {
  if (count < 1 || !jobs || !plan) return fail(ctx, DB200_ERR_INVALID, "rbf tiles: empty job list");
  std::vector<TileInst> host((size_t)count);
  int items = 0, nkc_max = 1, panel_max = 16, om_mult = 1;
  for (int b = 0; b < count; ++b) {
    const TileJob& J = jobs[b];
    const PackedPoints &pi = J.pi, &pj = J.pj;
    if (pi.dp != pj.dp || pi.dp > 128 || pi.dp % 32)
      return fail(ctx, DB200_ERR_UNSUPPORTED, "rbf tiles: padded feature count not in {32, 64, 96, 128}");
    if (pi.npad % PAIR_M || pj.npad % BN) return fail(ctx, DB200_ERR_INVALID, "rbf tiles: unpadded operands");
    const SketchPlan& P = J.plan;
    const int pcols = P.comp ? 128 : 64;  // P (and P_lo) columns of tensor memory
    if (mode == RBF_MODE_SKETCH && (P.panel % 16 || P.panel > 320 || P.panel < 16 || P.n_panels < 1 ||
                                    (P.g_bufs != 1 && P.g_bufs != 2) || P.panel + pcols + 128 * P.g_bufs > TMEM_COLS ||
                                    P.n_panels * P.panel < J.l || P.lrows < P.n_panels * P.panel ||
                                    P.comp < 0 || P.comp > 2 || (P.comp && P.panel > 256) || P.promote < 0 ||
                                    (P.comp == 2 && J.om_lo < P.lrows)))
      return fail(ctx, DB200_ERR_INVALID, "rbf tiles: bad sketch panel plan");
    TileInst& I = host[(size_t)b];
    std::memset(&I, 0, sizeof(I));
    const int kp = 2 * pi.dp;
    if (!make_tmap(&I.tm_xi, pi.xp, kp, pi.npad, kp, BM) || !make_tmap(&I.tm_xj, pj.xp, kp, pj.npad, kp, BN_HALF))
      return fail(ctx, DB200_ERR_CUDA, "cuTensorMapEncodeTiled failed for the point operands");
    if (mode == RBF_MODE_SKETCH) {
      I.n_panels = P.n_panels;
      I.panel = P.panel;
      // one sketch MMA of N = panel columns, or two of about half each (multiples of 16, each <= 256); each CTA
      // of the pair holds half of every instruction's B rows, loaded as one TMA box per instruction
      I.n1 = P.panel > 256 ? (P.panel / 32) * 16 : P.panel;
      I.n2 = P.panel - I.n1;
      // compensated (comp = 2): the lo rows of this job's panel columns start om_lo rows after its hi rows
      const int om_rows = (P.comp == 2) ? J.om_lo + P.lrows : P.lrows;
      if (!make_tmap(&I.tm_om1, J.op, pj.npad, om_rows, pj.npad, I.n1 / 2, CU_TENSOR_MAP_DATA_TYPE_FLOAT16) ||
          (I.n2 > 0 &&
           !make_tmap(&I.tm_om2, J.op, pj.npad, om_rows, pj.npad, I.n2 / 2, CU_TENSOR_MAP_DATA_TYPE_FLOAT16)))
        return fail(ctx, DB200_ERR_CUDA, "cuTensorMapEncodeTiled failed for the sketch operand");
      if (I.n2 == 0) I.tm_om2 = I.tm_om1;  // unused
      I.g_bufs = P.g_bufs;
      I.tmem_p = 128 * P.g_bufs;
      I.tmem_y = I.tmem_p + pcols;
      I.comp = P.comp;
      I.om_lo = (P.comp == 2) ? J.om_lo : 0;
      I.promote = P.promote;
      om_mult = std::max(om_mult, P.comp == 2 ? 2 : 1);
    } else {
      I.tm_om1 = I.tm_om2 = I.tm_xj;  // unused
      I.n_panels = 1;
      I.panel = 16;
      I.n1 = 16;
      I.n2 = 0;
      I.g_bufs = 2;
      I.tmem_p = 256;
      I.tmem_y = 320;
    }
    I.m = pi.n;
    I.n = pj.n;
    I.n_itiles = pi.npad / PAIR_M;
    I.n_jtiles = pj.npad / BN;
    I.l = J.l;
    I.nkc = kp / KC;
    I.c_row = -J.gamma * LOG2E;
    // UPDATE: gamma carries alpha; KNN: 1
    I.c_dot = (mode == RBF_MODE_UPDATE || mode == RBF_MODE_KNN) ? J.gamma : 2.0f * J.gamma * LOG2E;
    I.si = pi.norms;
    I.sj = pj.norms;
    // the pack writes the set's max |x|, its scale and whether any lo part is nonzero after the norms (a slice of a
    // packed set reads its parent's)
    const float* tail_i = pi.tail ? pi.tail : pi.norms + pi.npad;
    const float* tail_j = pj.tail ? pj.tail : pj.norms + pj.npad;
    I.fi = tail_i + 1;
    I.fj = tail_j + 1;
    I.lof_i = reinterpret_cast<const unsigned*>(tail_i + 2);
    I.lof_j = reinterpret_cast<const unsigned*>(tail_j + 2);
    I.yi = J.yi;
    I.yj = J.yj;
    I.out = J.out;
    I.ldo = J.ldo;
    I.item_begin = items;
    items += I.n_itiles * I.n_panels;
    nkc_max = std::max(nkc_max, I.nkc);
    panel_max = std::max(panel_max, I.panel);
  }
  TilePlan T;
  T.mode = mode;
  T.count = count;
  T.n_items = items;
  T.nkc_max = nkc_max;
  T.panel_max = panel_max;
  T.nso = (mode == RBF_MODE_SKETCH) ? MAX_NSO : 0;
  T.lean = (mode == RBF_MODE_SKETCH);
  for (int b = 0; b < count; ++b) T.lean = T.lean && host[(size_t)b].comp == 0 && host[(size_t)b].promote == 0;
  T.om_mult = om_mult;
  {  // the Xj ring takes whatever shared memory is left
    const SmemLayout L0 = make_layout(nkc_max, panel_max, 0, T.nso, om_mult);
    const long long left = (long long)SMEM_LIMIT - 1024 - (long long)L0.total;
    int nsx = (int)(left / XJ_CHUNK);
    if (nsx > MAX_NSX) nsx = MAX_NSX;
    if (nsx < 2) return fail(ctx, DB200_ERR_UNSUPPORTED, "rbf tiles: shared memory plan does not fit");
    T.nsx = nsx;
  }
  T.smem = make_layout(nkc_max, panel_max, T.nsx, T.nso, om_mult).total + 1024;
  {
    const int max_clusters = ctx->num_sms / 2;
    cudaError_t e =
        (mode == RBF_MODE_SKETCH)
            ? (T.lean ? plan_clusters<RBF_MODE_SKETCH, true>(T.smem, max_clusters, items, &T.clusters)
                      : plan_clusters<RBF_MODE_SKETCH, false>(T.smem, max_clusters, items, &T.clusters))
        : (mode == RBF_MODE_UPDATE) ? plan_clusters<RBF_MODE_UPDATE, false>(T.smem, max_clusters, items, &T.clusters)
        : (mode == RBF_MODE_KNN)    ? plan_clusters<RBF_MODE_KNN, false>(T.smem, max_clusters, items, &T.clusters)
                                    : plan_clusters<RBF_MODE_KBLOCK, false>(T.smem, max_clusters, items, &T.clusters);
    DB200_CUDA(ctx, e);
  }
  const size_t bytes = tile_table_bytes(count);
  void* d = table_storage;
  if (d) {
    if (table_capacity < bytes) return fail(ctx, DB200_ERR_TOO_LARGE, "rbf tiles: instance table storage too small");
  } else {
    if (bytes > ctx->tile_table_size) {
      DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      if (ctx->tile_table) cudaFree(ctx->tile_table);
      ctx->tile_table = nullptr;
      ctx->tile_table_size = 0;
      DB200_CUDA(ctx, cudaMalloc(&ctx->tile_table, bytes));
      ctx->tile_table_size = bytes;
    }
    d = ctx->tile_table;
  }
  // pageable source: the copy is staged before the call returns, so `host` may go out of scope
  DB200_CUDA(ctx, cudaMemcpyAsync(d, host.data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
  T.table = d;
  static_assert(sizeof(T.tm1) == 4 * sizeof(CUtensorMap), "tensor map copy");
  std::memcpy(T.tm1, &host[0].tm_xi, sizeof(T.tm1));
  *plan = T;
  return DB200_OK;
}

int launch_rbf_plan(db200_context* ctx, const TilePlan& T) {
  LaunchArgs a;
  std::memcpy(a.tm1, T.tm1, sizeof(a.tm1));
  a.inst = static_cast<const TileInst*>(T.table);
  a.count = T.count;
  a.n_items = T.n_items;
  a.nsx = T.nsx;
  a.nso = T.nso;
  a.om_mult = T.om_mult;
  a.nkc_max = T.nkc_max;
  a.panel_max = T.panel_max;
  a.status = ctx->d_status;
  cudaEvent_t e0 = nullptr;
  prof_begin(ctx, &e0);
  cudaError_t err =
      (T.mode == RBF_MODE_SKETCH)
          ? (T.lean ? launch_kernel<RBF_MODE_SKETCH, true>(a, T.smem, T.clusters, ctx->stream)
                    : launch_kernel<RBF_MODE_SKETCH, false>(a, T.smem, T.clusters, ctx->stream))
      : (T.mode == RBF_MODE_UPDATE) ? launch_kernel<RBF_MODE_UPDATE, false>(a, T.smem, T.clusters, ctx->stream)
      : (T.mode == RBF_MODE_KNN)    ? launch_kernel<RBF_MODE_KNN, false>(a, T.smem, T.clusters, ctx->stream)
                                    : launch_kernel<RBF_MODE_KBLOCK, false>(a, T.smem, T.clusters, ctx->stream);
  DB200_CUDA(ctx, err);
  prof_end(ctx, e0);
  count_launch(ctx);
  return DB200_OK;
}

int launch_rbf_tiles(db200_context* ctx, int mode, const PackedPoints& pi, const PackedPoints& pj, const float* yi,
                     const float* yj, const void* op, const SketchPlan& plan, int l, float gamma, float* out,
                     int ldo, void* table_storage, size_t table_capacity) {
  TileJob J;
  J.pi = pi;
  J.pj = pj;
  J.yi = yi;
  J.yj = yj;
  J.op = op;
  J.plan = plan;
  J.om_lo = plan.lrows;  // a compensated Omega~ packs its lo rows after all hi rows
  J.l = l;
  J.gamma = gamma;
  J.out = out;
  J.ldo = ldo;
  TilePlan T;
  int st = prepare_rbf_tiles(ctx, mode, &J, 1, table_storage, table_capacity, &T);
  if (st) return st;
  return launch_rbf_plan(ctx, T);
}

// A sketch wider than one panel as per-panel instances of exact widths: the padded width roundup(l, 16) split into
// plan.n_panels panels of multiples of 16 that differ by at most 16 columns (528 = 272 + 256 instead of 2 x 272),
// so no panel computes sketch columns past l beyond the last multiple of 16.  `base` carries the points, labels,
// packed Omega~ (plan.lrows hi rows, then as many lo rows when compensated) and the output.
void exact_panel_jobs(const TileJob& base, std::vector<TileJob>& out) {
  const SketchPlan& plan = base.plan;
  if (plan.n_panels <= 1) {
    TileJob J = base;
    J.om_lo = plan.lrows;
    out.push_back(J);
    return;
  }
  const int l = base.l, units = (l + 15) / 16, np = plan.n_panels;
  int off = 0;
  for (int p = 0; p < np; ++p) {
    const int w = 16 * (units / np + (p < units % np ? 1 : 0));
    TileJob J = base;
    J.op = static_cast<const uint16_t*>(base.op) + (size_t)off * base.pj.npad;  // packed rows = sketch columns
    J.plan.n_panels = 1;
    J.plan.panel = w;
    J.plan.lrows = w;
    J.plan.g_bufs = (w + (plan.comp ? 128 : 64) + 2 * 128 <= TMEM_COLS) ? 2 : 1;
    J.om_lo = plan.lrows;  // lo rows of the whole packed operand follow its plan.lrows hi rows
    J.l = std::min(w, l - off);
    J.out = base.out + (size_t)off * base.ldo;
    out.push_back(J);
    off += w;
  }
}

int launch_rbf_sketch_exact(db200_context* ctx, const PackedPoints& pi, const PackedPoints& pj, const float* yi,
                            const void* op, const SketchPlan& plan, int l, float gamma, float* out, int ldo) {
  TileJob base;
  base.pi = pi;
  base.pj = pj;
  base.yi = yi;
  base.yj = nullptr;  // folded into the packed Omega~
  base.op = op;
  base.plan = plan;
  base.l = l;
  base.gamma = gamma;
  base.out = out;
  base.ldo = ldo;
  std::vector<TileJob> jobs;
  exact_panel_jobs(base, jobs);
  TilePlan T;
  int st = prepare_rbf_tiles(ctx, RBF_MODE_SKETCH, jobs.data(), (int)jobs.size(), nullptr, 0, &T);
  if (st) return st;
  return launch_rbf_plan(ctx, T);
}

}  // namespace db200
