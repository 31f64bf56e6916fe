// Tensor-core (tcgen05) weighted Gram for the Woodbury capacity matrix of the Newton step:
//     M += Z~^T Z~,   Z~ = diag(sqrt(w)) Z   (Z: n x r FP64 column major, w = D^-1 >= 0)
// The operand is split into bf16 hi + lo (hi.hi + hi.lo + lo.hi, fp32 accumulation in TMEM, relative error of
// the products ~2^-16), the n dimension is split across CTAs and each CTA adds its 128 x 128 tile into the FP64
// matrix with FP64 atomics.  The barrier solver refines the resulting Newton step against the exact FP64
// operator (Z Z^T + D), so the tensor-core Gram only has to be a good preconditioner.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <mutex>

#include "internal.h"
#include "ptx.cuh"

namespace db200 {
namespace {

constexpr int TM = 128;                       // output tile (rows and columns of M)
constexpr int KCH = 64;                       // k chunk: 64 bf16 = one 128-byte swizzled row
constexpr int OPB = TM * KCH * 2;             // one operand chunk, 16 KB
constexpr int STAGE = 4 * OPB;                // Ahi, Alo, Bhi, Blo
constexpr int NSTAGE = 3;
constexpr int THREADS = 192;                  // warp 0 TMA, warp 1 MMA, warps 2..5 epilogue

struct GramArgs {
  int r;          // valid rows / columns of M
  int ntiles;     // tiles per side
  int kchunks;    // total k chunks (npad / 64)
  int chunks_per_split;
  double* M;
  int ldm;
  int* status;
};

__global__ void __launch_bounds__(THREADS, 1)
    gram_tc_kernel(const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo, GramArgs g) {
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

  // tile pair (upper triangle only) and k range of this CTA
  int tpair = blockIdx.x;
  int ti = 0;
  while (tpair >= g.ntiles - ti) {
    tpair -= g.ntiles - ti;
    ++ti;
  }
  const int tj = ti + tpair;
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
    tmem_alloc(smem_u32(tmem_slot), 128);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0 && nk > 0) {
      prefetch_tmap(&tm_hi);
      prefetch_tmap(&tm_lo);
      int issued = 0;
      for (int k = 0; k < nk; ++k, ++issued) {
        const int s = k % NSTAGE;
        const uint32_t ph = (k / NSTAGE) & 1;
        if (!mbar_wait(empty(s), ph ^ 1, abort_flag)) break;
        mbar_arrive_expect_tx(full(s), STAGE);
        const uint32_t base = s_op + s * STAGE;
        const int x = (k0 + k) * KCH;
        tma_load_2d(base + 0 * OPB, &tm_hi, full(s), x, ti * TM);
        tma_load_2d(base + 1 * OPB, &tm_lo, full(s), x, ti * TM);
        tma_load_2d(base + 2 * OPB, &tm_hi, full(s), x, tj * TM);
        tma_load_2d(base + 3 * OPB, &tm_lo, full(s), x, tj * TM);
      }
      if (*abort_flag) {
        volatile int never = 0;
        for (int k = (issued > NSTAGE ? issued - NSTAGE : 0); k < issued; ++k)
          mbar_wait(full(k % NSTAGE), (k / NSTAGE) & 1, &never);
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_f16(TM, TM, true);
      bool ok = true;
      for (int k = 0; k < nk && ok; ++k) {
        const int s = k % NSTAGE;
        if (!mbar_wait(full(s), (k / NSTAGE) & 1, abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t base = s_op + s * STAGE;
#pragma unroll
        for (int ks = 0; ks < KCH / 16; ++ks) {
          const uint64_t ahi = sdesc_k_sw128(base + 0 * OPB + ks * 32), alo = sdesc_k_sw128(base + 1 * OPB + ks * 32);
          const uint64_t bhi = sdesc_k_sw128(base + 2 * OPB + ks * 32), blo = sdesc_k_sw128(base + 3 * OPB + ks * 32);
          umma_f16(tmem, ahi, bhi, idesc, (k | ks) ? 1u : 0u);
          umma_f16(tmem, ahi, blo, idesc, 1u);
          umma_f16(tmem, alo, bhi, idesc, 1u);
        }
        umma_commit(empty(s));
      }
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
      for (int c0 = 0; c0 < TM; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + c0, v);
        tmem_wait_ld();
        if (row < g.r) {
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const int col = tj * TM + c0 + e;
            if (col < g.r && row <= col) atomicAdd(g.M + (long long)col * g.ldm + row, (double)v[e]);
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
    tmem_dealloc(tmem, 128);
  }
}

// Z~^T split into bf16 hi / lo, [rpad][npad] each: out[c][i] = sqrt(w_i) Z[i + c*ldz] (zero padding).
__global__ void pack_scaled_t_kernel(const double* __restrict__ Z, long long ldz, const double* __restrict__ w, int n,
                                     int r, int npad, int rpad, __nv_bfloat16* __restrict__ hi,
                                     __nv_bfloat16* __restrict__ lo) {
  const long long total = (long long)npad * rpad;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % npad), c = (int)(e / npad);
    float x = 0.f;
    if (i < n && c < r) x = (float)(sqrt(w ? w[i] : 1.0) * Z[i + (long long)c * ldz]);
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    hi[e] = h;
    lo[e] = __float2bfloat16_rn(x - __bfloat162float(h));
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

bool tmap_rows(CUtensorMap* tm, const void* base, uint64_t inner, uint64_t rows) {
  auto enc = encode_fn();
  if (!enc) return false;
  cuuint64_t dims[2] = {inner, rows};
  cuuint64_t strides[1] = {inner * 2};
  cuuint32_t box[2] = {KCH, TM};
  cuuint32_t estr[2] = {1, 1};
  return enc(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

size_t gram_tc_scratch_bytes(int n, int r) {
  const size_t npad = (size_t)round_up(n, KCH), rpad = (size_t)round_up(r, TM);
  return 2 * align_up(npad * rpad * 2, 256) + 512;
}

// M (upper triangle, FP64, r x r) += Z~^T Z~ with Z~ = diag(sqrt(w)) Z.  `scratch` holds gram_tc_scratch_bytes.
int gram_tc_weighted(db200_context* ctx, int n, int r, const double* Z, long long ldz, const double* w, double* M,
                     int ldm, void* scratch) {
  const int npad = round_up(n, KCH), rpad = round_up(r, TM);
  Carve cv{static_cast<char*>(scratch)};
  __nv_bfloat16* hi = cv.take<__nv_bfloat16>((size_t)npad * rpad);
  __nv_bfloat16* lo = cv.take<__nv_bfloat16>((size_t)npad * rpad);
  const long long total = (long long)npad * rpad;
  long long blocks = (total + 255) / 256;
  if (blocks > 16LL * ctx->num_sms) blocks = 16LL * ctx->num_sms;
  pack_scaled_t_kernel<<<(unsigned)blocks, 256, 0, ctx->stream>>>(Z, ldz, w, n, r, npad, rpad, hi, lo);
  DB200_CUDA(ctx, cudaGetLastError());
  count_launch(ctx);
  CUtensorMap thi, tlo;
  if (!tmap_rows(&thi, hi, npad, rpad) || !tmap_rows(&tlo, lo, npad, rpad))
    return fail(ctx, DB200_ERR_CUDA, "gram_tc: cuTensorMapEncodeTiled failed");
  GramArgs a;
  a.r = r;
  a.ntiles = rpad / TM;
  a.kchunks = npad / KCH;
  const int pairs = a.ntiles * (a.ntiles + 1) / 2;
  int splits = (2 * ctx->num_sms + pairs - 1) / pairs;
  if (splits > a.kchunks) splits = a.kchunks;
  if (splits < 1) splits = 1;
  a.chunks_per_split = (a.kchunks + splits - 1) / splits;
  splits = (a.kchunks + a.chunks_per_split - 1) / a.chunks_per_split;
  a.M = M;
  a.ldm = ldm;
  a.status = ctx->d_status;
  const size_t smem = NSTAGE * STAGE + 512 + 1024;
  DB200_CUDA(ctx, cudaFuncSetAttribute(gram_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(pairs, splits);
  cudaEvent_t e0 = nullptr;
  prof_begin(ctx, &e0);
  gram_tc_kernel<<<grid, THREADS, smem, ctx->stream>>>(thi, tlo, a);
  DB200_CUDA(ctx, cudaGetLastError());
  prof_end(ctx, e0);
  count_launch(ctx);
  return DB200_OK;
}

}  // namespace db200
