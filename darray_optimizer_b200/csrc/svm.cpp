// Host orchestration of the kernel-SVM path (C++ over the device kernels): dense FP64 LA entry points,
// CholeskyQR2, the Nystrom low-rank factor and the barrier / Newton loop.
//
// Restated from tests/testsvm.cpp:86-321 (the SVM driver), include/lapack_like.h:10-90,283-379 and
// include/dbarrier.h:14-139, with the corrections listed in oracle/oracle.py's header (every block of K, the
// Q C Q^T core, the Woodbury Newton system, a line search that keeps 0 < a < C, barrier stop at 1e-6).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "barrier.h"
#include "internal.h"
#include "la64.h"

namespace db200 {
namespace {

struct EventTimer {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaStream_t s;
  explicit EventTimer(cudaStream_t st) : s(st) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
  }
  double stop_ms() {
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms;
  }
  ~EventTimer() {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
};

// Device status pair [status, bad index] used by potrf; lives at the start of the LA slot.
struct LaStatus {
  int* d = nullptr;
};

// Scalar readbacks go through the context's pinned staging area: a copy into pageable memory is staged by the
// driver and, from several threads at once (the batched solve's workers), serialises them.
int read_scalar(db200_context* ctx, const double* d_src, double* out) {
  DB200_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, d_src, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *out = ctx->h_pinned[0];
  return DB200_OK;
}

int read_status(db200_context* ctx, int* d_pair, int* st, int* bad) {
  int* h = reinterpret_cast<int*>(ctx->h_pinned);
  DB200_CUDA(ctx, cudaMemcpyAsync(h, d_pair, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *st = h[0];
  *bad = h[1];
  return DB200_OK;
}

// All-reduce k <= 64 host values over the attached collective through device scratch d_tmp (k doubles).
int allreduce_host(db200_context* ctx, double* d_tmp, double* vals, int k, int op) {
  if (!sharded(ctx)) return DB200_OK;
  std::memcpy(ctx->h_pinned, vals, sizeof(double) * k);
  DB200_CUDA(ctx, cudaMemcpyAsync(d_tmp, ctx->h_pinned, sizeof(double) * k, cudaMemcpyHostToDevice, ctx->stream));
  int st = allreduce(ctx, d_tmp, k, op);
  if (st) return st;
  DB200_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, d_tmp, sizeof(double) * k, cudaMemcpyDeviceToHost, ctx->stream));
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::memcpy(vals, ctx->h_pinned, sizeof(double) * k);
  return DB200_OK;
}

// One CholeskyQR pass Yout = Yin R^-1 with R = chol(Yin^T Yin + shift I); returns NOT_SPD without touching Yout
// when the Gram is not positive definite.  W, Rinv: l x l scratch; R (l x l) receives the factor.
int cholqr_pass(db200_context* ctx, int n, int l, const double* Yin, int ldin, double* Yout, int ldout, double* R,
                double* Rinv, double shift_rel, int* d_pair, double* d_scalar, bool tc_gram, bool dist) {
  // Gram W = Y^T Y (upper triangle).  tc_gram: on the int8 tensor cores, 8 signed 7-bit digits per value, exact
  // integer products, error ~3e-14 of ||y_p|| ||y_q||; otherwise on the FP64 pipes.  The Cholesky stays FP64.
  int st = DB200_OK;
  if (tc_gram) {
    void* scratch = slot_buffer(ctx, SLOT_SPARE, gram_tc_scratch_bytes(n, l));
    if (!scratch) return DB200_ERR_NOMEM;
    DB200_CUDA(ctx, cudaMemsetAsync(R, 0, sizeof(double) * (size_t)l * l, ctx->stream));
    if ((st = gram_tc_weighted(ctx, n, l, Yin, ldin, nullptr, R, l, scratch, 8))) return st;
  } else if ((st = gram<double, double>(ctx, n, l, l, Yin, ldin, Yin, ldin, nullptr, 1.0, 0.0, R, l, true))) {
    return st;
  }
  // row-sharded: the Gram of all rows is the sum of the ranks' Grams (upper triangles; the lower one is never read)
  if (dist && (st = allreduce(ctx, R, (long long)l * l, DB200_REDUCE_SUM))) return st;
  if (shift_rel > 0.0) {
    // shift = shift_rel * trace(W)
    if ((st = trace(ctx, R, l, l, d_scalar))) return st;
    double tr = 0;
    if ((st = read_scalar(ctx, d_scalar, &tr))) return st;
    if ((st = mirror_upper(ctx, R, l, l))) return st;  // the Gram kernel formed the upper triangle only
    if ((st = symmetrize(ctx, R, l, l, shift_rel * tr))) return st;
  }
  DB200_CUDA(ctx, cudaMemsetAsync(d_pair, 0, 2 * sizeof(int), ctx->stream));
  if ((st = potrf_upper(ctx, R, l, l, d_pair, d_pair + 1))) return st;
  int pst = 0, bad = 0;
  if ((st = read_status(ctx, d_pair, &pst, &bad))) return st;
  if (pst) return fail(ctx, DB200_ERR_NOT_SPD, "CholeskyQR: Gram matrix not positive definite at row " +
                                                   std::to_string(bad));
  if ((st = trinv_upper(ctx, R, l, l, Rinv, l))) return st;
  return gemm_tall<double, double>(ctx, n, l, l, Yin, ldin, Rinv, l, false, 0.0, Yout, ldout);
}

}  // namespace

size_t cholqr2_slot_bytes(int n, int l) {
  // slot layout: [pair | scalar | T (n x l) | R1 | R2 | R3 | Rinv | Racc]
  const size_t ll = (size_t)l * l;
  return 1024 + align_up((size_t)n * l * 8, 256) + 5 * align_up(ll * 8, 256) + 1024;
}

int cholqr2_impl(db200_context* ctx, int n, int l, double* Y, int ldy, double* Rout, int ldr, bool tc_gram,
                 bool dist) {
  const size_t ll = (size_t)l * l;
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_LA, cholqr2_slot_bytes(n, l)));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  int* d_pair = cv.take<int>(4);
  double* d_scalar = cv.take<double>(4);
  double* T = cv.take<double>((size_t)n * l);
  double* R1 = cv.take<double>(ll);
  double* R2 = cv.take<double>(ll);
  double* R3 = cv.take<double>(ll);
  double* Rinv = cv.take<double>(ll);
  double* Racc = cv.take<double>(ll);
  int st = cholqr_pass(ctx, n, l, Y, ldy, T, n, R1, Rinv, 0.0, d_pair, d_scalar, tc_gram, dist);
  bool shifted = false;
  if (st == DB200_ERR_NOT_SPD) {
    // shifted CholeskyQR3 (Fukaya, Kannan, Nakatsukasa, Yamamoto, Yanagisawa 2020): first pass with
    // shift 11 (n l + l (l + 1)) u ||Y||^2, ||Y||_2^2 <= trace(Y^T Y); n counts the rows of every rank
    double rows = n;
    if (dist && (st = allreduce_host(ctx, d_scalar, &rows, 1, DB200_REDUCE_SUM))) return st;
    const double u = 1.1102230246251565e-16;
    const double rel = 11.0 * (rows * l + (double)l * (l + 1)) * u;
    st = cholqr_pass(ctx, n, l, Y, ldy, T, n, R1, Rinv, rel, d_pair, d_scalar, tc_gram, dist);
    shifted = true;
  }
  if (st) return st;
  // second pass T -> Y
  if ((st = cholqr_pass(ctx, n, l, T, n, Y, ldy, R2, Rinv, 0.0, d_pair, d_scalar, tc_gram, dist))) return st;
  // R = R2 R1 (upper * upper)
  if ((st = gemm_tall<double, double>(ctx, l, l, l, R2, l, R1, l, false, 0.0, Racc, l))) return st;
  if (shifted) {
    // third pass Y -> T, then copy back; R = R3 (R2 R1)
    if ((st = cholqr_pass(ctx, n, l, Y, ldy, T, n, R3, Rinv, 0.0, d_pair, d_scalar, tc_gram, dist))) return st;
    DB200_CUDA(ctx, cudaMemcpy2DAsync(Y, sizeof(double) * ldy, T, sizeof(double) * n, sizeof(double) * n, l,
                                      cudaMemcpyDeviceToDevice, ctx->stream));
    if ((st = gemm_tall<double, double>(ctx, l, l, l, R3, l, Racc, l, false, 0.0, R1, l))) return st;
    Racc = R1;
  }
  if (Rout) {
    DB200_CUDA(ctx, cudaMemcpy2DAsync(Rout, sizeof(double) * ldr, Racc, sizeof(double) * l, sizeof(double) * l, l,
                                      cudaMemcpyDeviceToDevice, ctx->stream));
  }
  return DB200_OK;
}

// ---------------------------------------------------------------------------------------------- barrier
namespace {

// The capacity matrix M = I + Z^T D^-1 Z of a Newton step and its first Cholesky attempt, as launches on
// ctx->stream only (so that the sequence can be captured in a graph): the Gram (int8 tensor cores, `slices`
// digits, or FP64), then the identity, the unshifted backup L = M, the status pair and potrf.
struct FactorSeq {
  const double* Z;
  int ldz;
  const double* dinv;
  double* M;
  double* L;
  int* d_pair;
  int n, r;
  bool use_tc;
  int slices;
  void* scratch;
};

int factor_gram(db200_context* ctx, const FactorSeq& f) {
  const size_t rr = (size_t)f.r * f.r;
  if (f.use_tc) {
    DB200_CUDA(ctx, cudaMemsetAsync(f.M, 0, sizeof(double) * rr, ctx->stream));
    return gram_tc_weighted(ctx, f.n, f.r, f.Z, f.ldz, f.dinv, f.M, f.r, f.scratch, f.slices);
  }
  return gram<double, double>(ctx, f.n, f.r, f.r, f.Z, f.ldz, f.Z, f.ldz, f.dinv, 1.0, 0.0, f.M, f.r, true);
}

int factor_tail(db200_context* ctx, const FactorSeq& f) {
  int st = bar_add_identity(ctx, f.M, f.r, f.r);
  if (st) return st;
  DB200_CUDA(ctx, cudaMemcpyAsync(f.L, f.M, sizeof(double) * (size_t)f.r * f.r, cudaMemcpyDeviceToDevice,
                                  ctx->stream));
  DB200_CUDA(ctx, cudaMemsetAsync(f.d_pair, 0, 2 * sizeof(int), ctx->stream));
  return potrf_upper(ctx, f.M, f.r, f.r, f.d_pair, f.d_pair + 1);
}

int factor_seq(db200_context* ctx, const FactorSeq& f) {
  int st = factor_gram(ctx, f);
  return st ? st : factor_tail(ctx, f);
}

// Class-balanced start (tests/testsvm.cpp:192-212) from the class counts.
void set_a0_counts(double plus, double minus, double C, double* pval, double* mval) {
  if (plus > minus) {
    *mval = 0.9 * C;
    *pval = minus > 0 ? *mval * minus / plus : *mval;
  } else {
    *pval = 0.9 * C;
    *mval = plus > 0 ? *pval * plus / minus : *pval;
  }
}

}  // namespace

size_t barrier_slot_bytes(int n, int r, bool mixed) {
  const size_t rr = (size_t)r * r;
  const size_t tc_bytes = mixed ? gram_tc_scratch_bytes(n, r) : 0;
  return 4096 + 10 * align_up((size_t)n * 8, 256) + 6 * align_up((size_t)r * 8, 256) + 2 * align_up(rr * 8, 256) +
         align_up(tc_bytes, 256) + 4096;
}

int svm_barrier_impl(db200_context* ctx, int n, int r, const double* Z, int ldz, const float* y, double C,
                     const db200_barrier_params& P, double* a, db200_svm_report* rep, bool dist) {
  if (r > 4096) return fail(ctx, DB200_ERR_UNSUPPORTED, "svm_barrier: r > 4096");
  EventTimer timer(ctx->stream);
  const size_t rr = (size_t)r * r;
  const bool mixed = (P.precision != DB200_FP64);
  const size_t tc_bytes = mixed ? gram_tc_scratch_bytes(n, r) : 0;
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_BAR, barrier_slot_bytes(n, r, mixed)));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  double* red = cv.take<double>(64);
  double* taus = cv.take<double>(16);
  double* ls = cv.take<double>(32);
  double* sc = cv.take<double>(8);  // scalars: [0] w.w, [1] w.v, [2] v.v, [3] hinge, [4..6] products with y
  int* d_pair = cv.take<int>(4);
  double* g = cv.take<double>(n);
  double* dinv = cv.take<double>(n);
  double* s = cv.take<double>(n);
  double* w = cv.take<double>(r);
  double* v = cv.take<double>(r);
  double* u = cv.take<double>(r);
  double* M = cv.take<double>(rr);
  double* L = cv.take<double>(rr);
  double* res = cv.take<double>(n);
  double* delta = cv.take<double>(n);
  double* zw = cv.take<double>(n);  // Z w for the current w = Z^T a (valid while zw_ok)
  double* zv = cv.take<double>(n);  // Z v for v = Z^T s, written by a refinement check
  double* yd = cv.take<double>(n);  // labels in FP64 (bias mode)
  double* sy = cv.take<double>(n);  // -H~^-1 y (bias mode)
  double* gb = cv.take<double>(n);  // g + nu y (bias mode)
  void* tc_scratch = mixed ? static_cast<void*>(cv.take<char>(tc_bytes)) : nullptr;
  int refine_total = 0, fallbacks_total = 0;
  // Tensor-core capacity matrix: 8 int8 digits per value (36 products, ~3e-14 of the column norms), after that
  // the FP64 capacity matrix.  From r = 2048 the Gram (n r^2) outweighs the refinement passes (n r) that a coarser
  // capacity matrix costs, so there the ladder starts at 6 digits (21 products, ~3e-10) while the refinement
  // converges with it.  (Measured: 6 digits first cut the barrier at n = 524288, r = 2064 from 8.6 to 7.3 s, and
  // lengthened it at r = 528 from 181 to 221 ms and at r = 1040 from 0.83 to 1.28 s.)
  constexpr int kSlices[2] = {6, 8};
  int tc_level = (r >= 2048) ? 0 : 1;  // index into kSlices; 2 = FP64
  bool tc_ok = true;
  int st0 = DB200_OK;

  // Reductions over rows: at one rank the kernels' own sums; row-sharded, all-reduced over the ranks (the
  // r-vectors Z^T x, the capacity matrix and the scalar sums, maxima and minima), so that every rank takes the same
  // decisions.
  auto reduce = [&](double* buf, long long count, int op) -> int {
    return dist ? allreduce(ctx, buf, count, op) : DB200_OK;
  };
  auto gemv_t = [&](const double* v, const double* scale, double sign, double* out) -> int {
    int s2 = bar_gemv_t(ctx, n, r, Z, ldz, v, scale, sign, out);
    return s2 ? s2 : reduce(out, r, DB200_REDUCE_SUM);
  };
  // red after bar_grad_hess: [0] sum a, [1] sum logs, [2] max D, [3] min D
  auto reduce_grad = [&]() -> int {
    int s2 = reduce(red, 2, DB200_REDUCE_SUM);
    if (!s2) s2 = reduce(red + 2, 1, DB200_REDUCE_MAX);
    return s2 ? s2 : reduce(red + 3, 1, DB200_REDUCE_MIN);
  };
  // A fixed launch sequence of a Newton step (its pointers and scalars are those of this call): at one rank it is
  // replayed from a CUDA graph, one launch instead of several per step; row-sharded it runs as it is, since its
  // all-reduces call back into the host.
  long long c_bits = 0, beta_bits = 0;
  std::memcpy(&c_bits, &C, sizeof(c_bits));
  std::memcpy(&beta_bits, &P.beta, sizeof(beta_bits));
  auto seq = [&](long long tag, std::initializer_list<long long> extra, const std::function<int()>& body) -> int {
    if (dist) return body();
    std::vector<long long> key = {tag, (long long)Z, ldz, n, r, (long long)base, (long long)a, c_bits, beta_bits};
    key.insert(key.end(), extra);
    return graph_run(ctx, key, body);
  };
  // out = -H~^-1 rhs by Woodbury on the factored capacity matrix; rd[0..2] <- its direction statistics
  auto woodbury_body = [&](const double* rhs, double* out, double* rd) -> int {
    int s2;
    if ((s2 = gemv_t(rhs, dinv, -1.0, u))) return s2;
    if ((s2 = trsv_upper(ctx, M, L, r, r, u, true))) return s2;   // R^T z = rhs
    if ((s2 = trsv_upper(ctx, M, L, r, r, u, false))) return s2;  // R u = z
    if ((s2 = bar_init_red(ctx, rd, 2, 0, 1))) return s2;
    return bar_direction(ctx, n, r, Z, ldz, u, rhs, dinv, a, C, out, rd);
  };
  auto woodbury = [&](const double* rhs, double* out, double* rd) -> int {
    return seq(1, {(long long)rhs, (long long)out, (long long)rd},
               [&]() -> int { return woodbury_body(rhs, out, rd); });
  };
  // red[16..17] <- |res|^2, |rhs|^2 of the Newton residual res = rhs + H out, with v = Z^T out and zv = Z v
  auto residual = [&](const double* rhs, double* out) -> int {
    return seq(2, {(long long)rhs, (long long)out}, [&]() -> int {
      int s2;
      if ((s2 = gemv_t(out, nullptr, 1.0, v))) return s2;
      if ((s2 = bar_init_red(ctx, red + 16, 2, 0, 0))) return s2;
      if ((s2 = bar_residual(ctx, n, r, Z, ldz, v, rhs, dinv, out, res, red + 16, zv))) return s2;
      return reduce(red + 16, 2, DB200_REDUCE_SUM);
    });
  };

  // class-balanced start (tests/testsvm.cpp:192-212) from the class counts of all rows
  std::vector<float> hy(n);
  DB200_CUDA(ctx, cudaMemcpyAsync(hy.data(), y, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream));
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  double counts[2] = {0.0, (double)n};  // [plus, rows]
  for (int i = 0; i < n; ++i) counts[0] += hy[i] == 1.0f;
  if (dist && (st0 = allreduce_host(ctx, red, counts, 2, DB200_REDUCE_SUM))) return st0;
  const double n_all = counts[1];  // rows of every rank
  double pval = 0, mval = 0;
  set_a0_counts(counts[0], n_all - counts[0], C, &pval, &mval);
  {
    std::vector<double> ha(n), hyd(n);
    for (int i = 0; i < n; ++i) {
      ha[i] = (hy[i] == 1.0f) ? pval : mval;
      hyd[i] = (hy[i] == 1.0f) ? 1.0 : -1.0;
    }
    if (P.bias && (counts[0] == 0 || counts[0] == n_all))
      return fail(ctx, DB200_ERR_INFEASIBLE, "svm_barrier: the bias needs both classes (y^T a = 0)");
    DB200_CUDA(ctx, cudaMemcpyAsync(a, ha.data(), sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    if (P.bias)
      DB200_CUDA(ctx, cudaMemcpyAsync(yd, hyd.data(), sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  double bias_nu = 0.0;  // multiplier of y^T a = 0 at the last Newton step (the decision function's bias)

  double t = P.t0;
  int total_newton = 0, outer = 0, status = DB200_OK;
  double prev_pd = -1.0;  // primal-dual gap at the previous outer step whose barrier bound was met
  double h[64];
  int st;
  auto fetch = [&](const double* d_src, int count) -> int {  // count <= 64 (pinned staging holds 512)
    DB200_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, d_src, sizeof(double) * count, cudaMemcpyDeviceToHost,
                                    ctx->stream));
    DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::memcpy(h, ctx->h_pinned, sizeof(double) * count);
    return DB200_OK;
  };
  double fa = 0.0, suma_now = 0.0;
  // In the mixed path an accepted step a += tau s with v = Z^T s and zv = Z v both current (a converged refinement
  // check) updates w += tau v and zw += tau zv, which saves the two passes over Z that recompute them; the
  // outer step's stop test recomputes both from a.
  bool zw_ok = false;
  // Capacity matrix M = I + Z^T D^-1 Z of the current D and its first Cholesky attempt (status in d_pair), enqueued
  // only: the caller reads the status.
  auto factor_launch = [&](bool use_tc) -> int {
    const FactorSeq fs{Z, ldz, dinv, M, L, d_pair, n, r, use_tc, kSlices[tc_level], tc_scratch};
    int s2;
    if (!dist) {
      // Gram, identity, backup, first Cholesky: one graph replay per Newton step (about 17 launches as separate
      // calls, which the host's launch path serialises when many solves share the GPU)
      const std::vector<long long> key = {(long long)Z, ldz, (long long)dinv, (long long)M, (long long)L,
                                          (long long)d_pair, n, r, use_tc ? fs.slices : 0, (long long)tc_scratch};
      return graph_run(ctx, key, [&]() -> int { return factor_seq(ctx, fs); });
    }
    if ((s2 = factor_gram(ctx, fs))) return s2;
    if ((s2 = reduce(M, (long long)rr, DB200_REDUCE_SUM))) return s2;  // upper triangles summed
    return factor_tail(ctx, fs);
  };
  // The first direction attempt of a Newton step factors its capacity matrix before the gradient statistics are
  // read back, so that one readback returns both: pre_status holds that factorisation's status for factor().
  bool prefactored = false, pre_tc = false;
  int pre_status = 0;
  for (outer = 1; outer <= P.max_outer; ++outer) {
    int ni = 0;
    while (true) {
      ++ni;
      ++total_newton;
      // gradient / Hessian diagonal at a
      if (zw_ok) {
        if ((st = bar_init_red(ctx, red, 2, 1, 1))) return st;
        if ((st = bar_grad_hess(ctx, n, r, Z, ldz, w, a, C, t, g, dinv, red, zw, nullptr))) return st;
      } else {
        if ((st = gemv_t(a, nullptr, 1.0, w))) return st;
        if ((st = bar_init_red(ctx, red, 2, 1, 1))) return st;
        if ((st = bar_grad_hess(ctx, n, r, Z, ldz, w, a, C, t, g, dinv, red, nullptr, zw))) return st;
        zw_ok = true;
      }
      pre_tc = mixed && tc_ok;
      if ((st = factor_launch(pre_tc))) return st;
      // the row reductions, w.w and the Cholesky status into red[0..13) for one readback
      if ((st = seq(5, {}, [&]() -> int {
             int s2;
             if ((s2 = reduce_grad()) || (s2 = bar_dot(ctx, r, w, w, sc))) return s2;
             DB200_CUDA(ctx, cudaMemcpyAsync(red + 8, sc, sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
             DB200_CUDA(ctx, cudaMemcpyAsync(red + 12, d_pair, 2 * sizeof(int), cudaMemcpyDeviceToDevice,
                                             ctx->stream));
             return DB200_OK;
           })))
        return st;
      if ((st = fetch(red, 13))) return st;
      const double suma = h[0], sumlog = h[1], dmax = h[2], dmin = h[3], ww = h[8];
      std::memcpy(&pre_status, &h[12], sizeof(int));
      prefactored = true;
      if (dmax / dmin > 1e18) break;  // tests/testsvm.cpp:258-263 (the factorisation above goes unused)
      const double lastg = 0.5 * ww - suma - sumlog / t;
      // Newton direction s = -(Z Z^T + D)^-1 g by Woodbury.  Mixed: capacity matrix M = I + Z^T D^-1 Z on the
      // int8 tensor cores (Ozaki slices, ~1e-12 of the column norms) factored in FP64, then iterative refinement
      // against the exact FP64 operator
      // until the relative residual is <= 1e-10; a step that does not get there is recomputed with the FP64
      // capacity matrix.  FP64: the capacity matrix on the FP64 pipes, no refinement.
      bool v_current = false;  // v already holds Z^T s (set by a converged refinement check)
      // Capacity matrix M = I + Z^T D^-1 Z and its Cholesky factor (upper in M, its transpose in L).
      auto factor = [&](bool use_tc) -> int {
        int s2;
        // A capacity matrix with a huge dynamic range (late in the barrier D^-1 spans ~18 orders) can sit on the
        // edge of numerical positive definiteness: its last bits (the Gram's rounding and the order of its
        // split-k additions) decide whether the FP64 Cholesky passes.  A relative diagonal shift, x10 from 1e-11 up
        // to 1 until the Cholesky succeeds, keeps it positive definite; the shifted M still gives a descent
        // direction, which the mixed path's refinement corrects against the exact operator.  L keeps the
        // unshifted M for the retries.
        int pst = 0, bad = 0;
        if (prefactored && use_tc == pre_tc) {
          pst = pre_status;  // factored before the gradient readback
        } else {
          if ((s2 = factor_launch(use_tc))) return s2;
          if ((s2 = read_status(ctx, d_pair, &pst, &bad))) return s2;
        }
        prefactored = false;
        double eps = 1e-11;
        for (int tries = 0;; ++tries) {
          if (tries > 0 && (s2 = read_status(ctx, d_pair, &pst, &bad))) return s2;
          if (pst == 0 || tries == 11) break;
          DB200_CUDA(ctx, cudaMemcpyAsync(M, L, sizeof(double) * rr, cudaMemcpyDeviceToDevice, ctx->stream));
          if ((s2 = bar_scale_diag(ctx, M, r, r, 1.0 + eps))) return s2;
          eps *= 10.0;
          DB200_CUDA(ctx, cudaMemsetAsync(d_pair, 0, 2 * sizeof(int), ctx->stream));
          if ((s2 = potrf_upper(ctx, M, r, r, d_pair, d_pair + 1))) return s2;
        }
        return transpose64(ctx, M, r, r, r, L, r);
      };
      // out = -(Z Z^T + D)^-1 rhs by Woodbury on the factored capacity matrix.  With the tensor-core capacity
      // matrix, iterative refinement against the exact FP64 operator (out += H~^-1 (-rhs - H out)) until the
      // relative residual is <= 1e-10; *converged reports whether it got there.  track_v: a converged check
      // leaves v = Z^T out and zv = Z v current.
      auto solve = [&](const double* rhs, double* out, bool use_tc, bool* converged, bool track_v) -> int {
        int s2;
        *converged = true;
        if ((s2 = woodbury(rhs, out, red))) return s2;
        if (!use_tc) return DB200_OK;
        *converged = false;
        double prev = 0.0;
        for (int it = 0; it <= P.refine_max; ++it) {
          if ((s2 = residual(rhs, out))) return s2;
          if ((s2 = fetch(red + 16, 2))) return s2;
          const double rn = std::sqrt(h[0]), gn = std::sqrt(h[1]);
          if (rn <= 1e-10 * gn) {
            *converged = true;
            if (track_v) v_current = true;  // v = Z^T out for the final out: the line search reuses it
            break;
          }
          if (it == P.refine_max || (it > 0 && rn >= 0.5 * prev) || !std::isfinite(rn)) break;
          prev = rn;
          if ((s2 = seq(3, {(long long)out}, [&]() -> int {  // out += -H~^-1 res
                 int s3 = woodbury_body(res, delta, red + 16);
                 return s3 ? s3 : bar_axpy(ctx, n, 1.0, delta, out);
               })))
            return s2;
          ++refine_total;
        }
        return DB200_OK;
      };
      // out = -H~^-1 rhs: one Woodbury application of the factored capacity matrix, no refinement.
      auto apply = [&](const double* rhs, double* out, double* rd) -> int { return woodbury(rhs, out, rd); };
      // Newton direction s = -(Z Z^T + D)^-1 g.  Mixed: capacity matrix on the int8 tensor cores (Ozaki slices,
      // ~1e-12 of the column norms) factored in FP64, then refinement; a step whose refinement misses 1e-10 is
      // recomputed with the FP64 capacity matrix.  FP64: the capacity matrix on the FP64 pipes, no refinement.
      //
      // With the bias, the bordered system [H y; y^T 0][s; nu] = [-g; 0].  With s~_y = -H~^-1 y (one more
      // application of the same factor): s = -H~^-1 g + nu s~_y with nu = -(y.s)/(y.s~_y) solves it for H~, and
      // refinement on the bordered system reuses s~_y, each step one application like the unbordered refinement:
      // res = g + nu y + H s, delta = -H~^-1 res, dnu = -(y.(s + delta))/(y.s~_y), s += delta + dnu s~_y,
      // nu += dnu.  Every iterate keeps y^T s = 0, so the iterates keep y^T a = 0.
      auto newton_dir = [&](bool use_tc, bool* converged) -> int {
        int s2;
        if ((s2 = factor(use_tc))) return s2;
        if (!P.bias) {
          if ((s2 = solve(g, s, use_tc, converged, true))) return s2;
          if (!use_tc) return DB200_OK;  // bar_direction's statistics stand
          if ((s2 = bar_init_red(ctx, red, 2, 0, 1))) return s2;
          return bar_step_stats(ctx, n, g, s, a, C, red);
        }
        *converged = true;
        if ((s2 = apply(g, s, red))) return s2;
        if ((s2 = apply(yd, sy, red + 16))) return s2;
        if ((s2 = bar_dot(ctx, n, yd, s, sc + 4))) return s2;
        if ((s2 = bar_dot(ctx, n, yd, sy, sc + 5))) return s2;
        if ((s2 = reduce(sc + 4, 2, DB200_REDUCE_SUM))) return s2;
        if ((s2 = fetch(sc + 4, 2))) return s2;
        const double ysy = h[1];
        if (ysy == 0.0 || !std::isfinite(ysy))
          return fail(ctx, DB200_ERR_NOT_SPD, "svm_barrier: bordered Newton system singular (y^T H^-1 y = 0)");
        double nu = -h[0] / ysy;
        if ((s2 = bar_axpy(ctx, n, nu, sy, s))) return s2;
        if (use_tc) {
          *converged = false;
          double prev = 0.0;
          for (int it = 0; it <= P.refine_max; ++it) {
            DB200_CUDA(ctx, cudaMemcpyAsync(gb, g, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
            if ((s2 = bar_axpy(ctx, n, nu, yd, gb))) return s2;
            if ((s2 = gemv_t(s, nullptr, 1.0, v))) return s2;
            if ((s2 = bar_init_red(ctx, red + 16, 2, 0, 0))) return s2;
            if ((s2 = bar_residual(ctx, n, r, Z, ldz, v, gb, dinv, s, res, red + 16, zv))) return s2;
            if ((s2 = reduce(red + 16, 2, DB200_REDUCE_SUM))) return s2;
            if ((s2 = fetch(red + 16, 2))) return s2;
            const double rn = std::sqrt(h[0]), gn = std::sqrt(h[1]);
            if (rn <= 1e-10 * gn) {
              *converged = true;
              v_current = true;  // v = Z^T s and zv = Z v for the final s
              break;
            }
            if (it == P.refine_max || (it > 0 && rn >= 0.5 * prev) || !std::isfinite(rn)) break;
            prev = rn;
            if ((s2 = apply(res, delta, red + 16))) return s2;
            if ((s2 = bar_axpy(ctx, n, 1.0, delta, s))) return s2;
            if ((s2 = bar_dot(ctx, n, yd, s, sc + 6))) return s2;
            if ((s2 = reduce(sc + 6, 1, DB200_REDUCE_SUM))) return s2;
            if ((s2 = fetch(sc + 6, 1))) return s2;
            const double dnu = -h[0] / ysy;
            if ((s2 = bar_axpy(ctx, n, dnu, sy, s))) return s2;
            nu += dnu;
            ++refine_total;
          }
        }
        bias_nu = nu;
        if ((s2 = bar_init_red(ctx, red, 2, 0, 1))) return s2;
        return bar_step_stats(ctx, n, g, s, a, C, red);
      };
      bool conv = true;
      v_current = false;
      if ((st = newton_dir(mixed && tc_ok, &conv))) return st;
      if (mixed && tc_ok && !conv && tc_level == 0) {
        // the barrier's D only grows more ill-conditioned with t: once the 6-digit capacity matrix no longer
        // preconditions well enough, this and the remaining Newton steps take the 8-digit one
        tc_level = 1;
        v_current = false;
        if ((st = newton_dir(true, &conv))) return st;
      }
      if (mixed && tc_ok && !conv) {
        // ... and once that misses the tolerance too, the FP64 capacity matrix
        ++fallbacks_total;
        tc_ok = false;
        tc_level = 2;
        v_current = false;
        if ((st = newton_dir(false, &conv))) return st;
      }
      // v = Z^T s (unless current), the direction statistics of s ([0] g.s, [1] sum s, [2] largest step inside
      // the box), w.v, v.v and the Cholesky status in red[0..13), and the line search's first 16 candidates,
      // tau_k = min(1, 0.99 step_max) beta^k formed on the device from red[2], their barrier sums in red[32..64):
      // one readback
      const bool need_v = !v_current;
      if ((st = seq(4, {need_v ? 1 : 0}, [&]() -> int {
             int s2;
             if (need_v && (s2 = gemv_t(s, nullptr, 1.0, v))) return s2;
             if ((s2 = reduce(red, 2, DB200_REDUCE_SUM)) || (s2 = reduce(red + 2, 1, DB200_REDUCE_MIN))) return s2;
             if ((s2 = bar_dot(ctx, r, w, v, sc + 1))) return s2;
             if ((s2 = bar_dot(ctx, r, v, v, sc + 2))) return s2;
             DB200_CUDA(ctx, cudaMemcpyAsync(red + 8, sc + 1, 2 * sizeof(double), cudaMemcpyDeviceToDevice,
                                             ctx->stream));
             DB200_CUDA(ctx, cudaMemcpyAsync(red + 12, d_pair, 2 * sizeof(int), cudaMemcpyDeviceToDevice,
                                             ctx->stream));
             if ((s2 = bar_steps16(ctx, red + 2, P.beta, taus))) return s2;
             if ((s2 = bar_linesearch16(ctx, n, a, s, C, taus, ls))) return s2;
             if ((s2 = reduce(ls, 32, DB200_REDUCE_SUM))) return s2;
             DB200_CUDA(ctx, cudaMemcpyAsync(red + 32, ls, 32 * sizeof(double), cudaMemcpyDeviceToDevice,
                                             ctx->stream));
             return DB200_OK;
           })))
        return st;
      if ((st = fetch(red, 64))) return st;
      int pst;
      std::memcpy(&pst, &h[12], sizeof(int));
      if (pst) return fail(ctx, DB200_ERR_NOT_SPD, "svm_barrier: Woodbury capacity matrix not positive definite");
      const double gs = h[0], sums = h[1], tmax = h[2], wv = h[8], vv = h[9];
      const double lam2 = -gs;
      // backtracking line search inside the box, 16 candidates per device pass; the first pass ran above with the
      // same candidates (formed by the same multiplications as here)
      double tau = std::min(1.0, 0.99 * tmax);
      double accepted = -1.0, newg = lastg;
      for (int sweep = 0; sweep < 4 && accepted < 0; ++sweep) {
        double ht[16];
        for (int k = 0; k < 16; ++k) {
          ht[k] = tau;
          tau *= P.beta;
        }
        const double* hl = h + 32;  // the first pass: read back with the step statistics
        if (sweep > 0) {
          // through the pinned staging area (past the readback slots): an asynchronous copy, which the fetch
          // below completes before the next sweep writes the slots again
          double* h_taus = ctx->h_pinned + 256;
          std::memcpy(h_taus, ht, sizeof(ht));
          DB200_CUDA(ctx, cudaMemcpyAsync(taus, h_taus, sizeof(ht), cudaMemcpyHostToDevice, ctx->stream));
          if ((st = bar_linesearch16(ctx, n, a, s, C, taus, ls))) return st;
          if ((st = reduce(ls, 32, DB200_REDUCE_SUM))) return st;
          if ((st = fetch(ls, 32))) return st;
          hl = h;
        }
        for (int k = 0; k < 16; ++k) {
          if (hl[16 + k] != 0.0) continue;  // leaves the box
          const double tk = ht[k];
          const double fk = 0.5 * (ww + 2.0 * tk * wv + tk * tk * vv) - (suma + tk * sums) - hl[k] / t;
          if (fk <= lastg + P.alpha * tk * gs) {
            accepted = tk;
            newg = fk;
            break;
          }
        }
      }
      if (accepted < 0) accepted = 0.0;  // no decrease found: stop this Newton loop below
      if (accepted > 0) {
        if ((st = bar_axpy(ctx, n, accepted, s, a))) return st;
        if (v_current) {
          if ((st = bar_axpy(ctx, r, accepted, v, w))) return st;
          if ((st = bar_axpy(ctx, n, accepted, zv, zw))) return st;
        } else {
          zw_ok = false;
        }
      }
      if (lam2 / 2 < P.newton_tol) break;
      if (accepted == 0.0) break;
      if (ni > 1 && (lastg - newg) < 1e-9 * std::fabs(newg)) break;
      if (ni >= P.max_newton) {
        status = DB200_ERR_MAXITER;
        break;
      }
    }
    // f(a) for the barrier stop
    if ((st = gemv_t(a, nullptr, 1.0, w))) return st;
    if ((st = bar_init_red(ctx, red, 2, 1, 1))) return st;
    if ((st = bar_grad_hess(ctx, n, r, Z, ldz, w, a, C, t, g, dinv, red, nullptr, zw))) return st;
    if ((st = reduce_grad())) return st;
    zw_ok = true;
    if ((st = bar_dot(ctx, r, w, w, sc))) return st;
    DB200_CUDA(ctx, cudaMemcpyAsync(red + 8, sc, sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    if ((st = fetch(red, 9))) return st;
    suma_now = h[0];
    fa = 0.5 * h[8] - suma_now;
    if (2.0 * n_all / t < P.gap_tol * std::fabs(fa)) {
      // The barrier bound is met.  Stop once the true primal-dual gap at w = Z^T a is within tolerance too, or
      // when a further outer step no longer halves it (it is then limited by the conditioning of the Newton
      // systems at large t, not by t: the plain-FP64 barrier stalls at the same gap, and a 10^6-fold tighter inner
      // Newton stop does not move it).
      if ((st = bar_dot(ctx, r, w, w, sc))) return st;
      if ((st = bar_hinge(ctx, n, r, Z, ldz, w, sc + 3, P.bias ? yd : nullptr, bias_nu))) return st;
      if ((st = reduce(sc + 3, 1, DB200_REDUCE_SUM))) return st;
      if ((st = fetch(sc, 4))) return st;
      const double pd = (0.5 * h[0] + C * h[3] + fa) / std::fabs(fa);
      if (pd < P.gap_tol || (prev_pd >= 0 && pd > 0.5 * prev_pd)) break;
      prev_pd = pd;
    }
    t *= P.mu;
  }
  if (outer > P.max_outer) {
    outer = P.max_outer;
    status = DB200_ERR_MAXITER;
  }
  // primal-dual gap at w = Z^T a (w is current), with the bias when the dual carries y^T a = 0
  if ((st = bar_hinge(ctx, n, r, Z, ldz, w, sc + 3, P.bias ? yd : nullptr, bias_nu))) return st;
  if ((st = reduce(sc + 3, 1, DB200_REDUCE_SUM))) return st;
  if ((st = fetch(sc, 4))) return st;
  const double primal = 0.5 * h[0] + C * h[3];
  if (rep) {
    rep->f = fa;
    rep->t = t;
    rep->outer = outer;
    rep->newton = total_newton;
    rep->gap_barrier = 2.0 * n_all / t / std::fabs(fa);
    rep->gap_primal_dual = (primal + fa) / std::fabs(fa);
    rep->status = status;
    rep->refine = refine_total;
    rep->fallbacks = fallbacks_total;
    rep->b = P.bias ? bias_nu : 0.0;
    rep->ms_barrier = timer.stop_ms();
  }
  return status == DB200_ERR_MAXITER ? DB200_ERR_MAXITER : DB200_OK;
}

// ---------------------------------------------------------------------------------------------- low rank
template <typename TY>
int nystrom_core(db200_context* ctx, int n, int l, const double* Q, const TY* Yk, double* Cm, double* R, int* d_pair,
                 double* d_scalar, double* Z, int ldz, double* nu_out, bool dist) {
  // C = Q^T (K Q), symmetrised; R^T R = C + nu I with nu = 1e-7 trace(C)/l, x10 until positive definite
  int st = gram<double, TY>(ctx, n, l, l, Q, n, Yk, n, nullptr, 1.0, 0.0, Cm, l, false);
  if (st) return st;
  if (dist && (st = allreduce(ctx, Cm, (long long)l * l, DB200_REDUCE_SUM))) return st;
  if ((st = symmetrize(ctx, Cm, l, l, 0.0))) return st;
  if ((st = trace(ctx, Cm, l, l, d_scalar))) return st;
  double tr = 0;
  if ((st = read_scalar(ctx, d_scalar, &tr))) return st;
  const size_t ll = (size_t)l * l;
  double nu = 1e-7 * std::max(tr, 1e-300) / l;
  bool ok = false;
  for (int tries = 0; tries < 12 && !ok; ++tries) {
    DB200_CUDA(ctx, cudaMemcpyAsync(R, Cm, sizeof(double) * ll, cudaMemcpyDeviceToDevice, ctx->stream));
    if ((st = symmetrize(ctx, R, l, l, nu))) return st;
    DB200_CUDA(ctx, cudaMemsetAsync(d_pair, 0, 2 * sizeof(int), ctx->stream));
    if ((st = potrf_upper(ctx, R, l, l, d_pair, d_pair + 1))) return st;
    int pst = 0, bad = 0;
    if ((st = read_status(ctx, d_pair, &pst, &bad))) return st;
    if (pst == 0) ok = true;
    else nu *= 10.0;
  }
  if (!ok) return fail(ctx, DB200_ERR_NOT_SPD, "lowrank: Q^T K Q + nu I not positive definite after 12 shifts");
  // Z = Q R^T
  if ((st = gemm_tall<double, double>(ctx, n, l, l, Q, n, R, l, true, 0.0, Z, ldz))) return st;
  if (nu_out) *nu_out = nu;
  return DB200_OK;
}
template int nystrom_core<float>(db200_context*, int, int, const double*, const float*, double*, double*, int*,
                                 double*, double*, int, double*, bool);
template int nystrom_core<double>(db200_context*, int, int, const double*, const double*, double*, double*, int*,
                                  double*, double*, int, double*, bool);

int lowrank_impl(db200_context* ctx, int n, int d, int l, int q, const float* X, int ldx, const float* y,
                 const float* Omega, int ldo, float gamma, int precision, double* Z, int ldz, db200_svm_report* rep,
                 bool dist) {
  if (l > n) return fail(ctx, DB200_ERR_INVALID, "lowrank: l > n");
  const bool fp64 = (precision == DB200_FP64);
  // this rank's rows [s0, s0 + m) of Y, Q and Z (all n rows at one rank)
  int s0 = 0, m = n;
  if (dist) {
    db200_row_shard(n, ctx->coll_world, ctx->coll_rank, &s0, &m);
    if (m < 1) return fail(ctx, DB200_ERR_INVALID, "lowrank: fewer points than ranks");
  }
  const float* Xi = X + (size_t)s0 * ldx;
  const float* yi = y + s0;
  const size_t ml = (size_t)m * l, nl = (size_t)n * l, ll = (size_t)l * l;
  // Qg: all rows of Q (FP64) for the next pass, gathered from the ranks; at one rank Q itself is complete
  const size_t bytes = 4096 + align_up(ml * 4, 256) + align_up(nl * 4, 256) + 2 * align_up(ml * 8, 256) +
                       (dist ? align_up(nl * 8, 256) : 0) + 3 * align_up(ll * 8, 256) + 4096;
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_PIPE, bytes));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  int* d_pair = cv.take<int>(4);
  double* d_scalar = cv.take<double>(4);
  float* Y32 = cv.take<float>(ml);  // mixed: kernel-pass output (fp32 accumulation)
  float* Qf = cv.take<float>(nl);   // mixed: all rows of Q as the next pass's test matrix
  double* Q = cv.take<double>(ml);
  double* Y64 = cv.take<double>(ml);  // FP64: kernel-pass output
  double* Qg = dist ? cv.take<double>(nl) : Q;
  double* Cm = cv.take<double>(ll);
  double* R = cv.take<double>(ll);
  double ms_sketch = 0, ms_orth = 0, ms_core = 0;
  int st;

  // one pass Y = diag(y) K diag(y) Om over this rank's rows, into Y32 (mixed) or Y64 (FP64).  Mixed: the compensated
  // sketch product with promoted accumulation; the range-finder passes (whose subspace, not scale, matters) in
  // 1024-point chunks, the final pass, whose Y scales the core C = Q^T K Q, in 256-point chunks.  Measured
  // dual-objective distance from the FP64 path: 5e-7 at n = 4096 (1.6e-6 with coarse chunks in the final pass) and
  // 4e-7 at n = 131072
  auto sketch_f32 = [&](const float* Om, int ldom, bool final_pass) -> int {
    EventTimer tm(ctx->stream);
    const int product = precision == DB200_MIXED_FAST ? DB200_SKETCH_SINGLE
                        : final_pass                  ? DB200_SKETCH_COMPENSATED_PROMOTED
                                                      : DB200_SKETCH_COMPENSATED_PROMOTED_COARSE;
    int s2 = db200_rbf_sketch_ex(ctx, m, n, d, l, Xi, ldx, X, ldx, DB200_POINT_MAJOR, yi, y, Om, ldom, Y32, m, gamma,
                                 product);
    ms_sketch += tm.stop_ms();
    return s2;
  };
  auto sketch_f64 = [&](const double* Om, int ldom) -> int {
    EventTimer tm(ctx->stream);
    int s2 = db200_rbf_sketch_f64(ctx, m, n, d, l, Xi, ldx, X, ldx, yi, y, Om, ldom, Y64, m, gamma);
    ms_sketch += tm.stop_ms();
    return s2;
  };
  auto orth = [&]() -> int {
    EventTimer tm(ctx->stream);
    int s2 = fp64 ? DB200_OK : convert<float, double>(ctx, Y32, m, Q, m, m, l);
    if (!s2 && fp64)
      s2 = (cudaMemcpyAsync(Q, Y64, sizeof(double) * ml, cudaMemcpyDeviceToDevice, ctx->stream) == cudaSuccess)
               ? DB200_OK
               : DB200_ERR_CUDA;
    // int8 Grams from n = 65536 (C2: CholeskyQR2 35 -> 28 ms, C3 207 -> 160 ms); below, the slicing's fixed
    // cost outweighs the FP64 Gram.  Decided on the global n, the same at every rank.
    if (!s2) s2 = cholqr2_impl(ctx, m, l, Q, m, nullptr, 0, !fp64 && n >= 65536, dist);
    if (!s2 && dist) {
      // all rows of Q: each rank's block at its offset in a zero matrix, summed over the ranks
      if (cudaMemsetAsync(Qg, 0, sizeof(double) * nl, ctx->stream) != cudaSuccess ||
          cudaMemcpy2DAsync(Qg + s0, sizeof(double) * n, Q, sizeof(double) * m, sizeof(double) * m, l,
                            cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess)
        s2 = cuda_fail(ctx, cudaGetLastError(), "lowrank: gather Q");
      if (!s2) s2 = allreduce(ctx, Qg, (long long)nl, DB200_REDUCE_SUM);
    }
    if (!s2 && !fp64) s2 = convert<double, float>(ctx, Qg, n, Qf, n, n, l);
    ms_orth += tm.stop_ms();
    return s2;
  };
  if (fp64) {
    // the FP64 comparator takes Omega in FP64 (all rows, in Qg: Q itself at one rank)
    if ((st = convert<float, double>(ctx, Omega, ldo, Qg, n, n, l))) return st;
    if ((st = sketch_f64(Qg, n))) return st;
  } else {
    if ((st = sketch_f32(Omega, ldo, false))) return st;
  }
  if ((st = orth())) return st;
  for (int it = 0; it < q; ++it) {
    if ((st = fp64 ? sketch_f64(Qg, n) : sketch_f32(Qf, n, false))) return st;
    if ((st = orth())) return st;
  }
  if ((st = fp64 ? sketch_f64(Qg, n) : sketch_f32(Qf, n, true))) return st;  // Y = K Q (this rank's rows)
  EventTimer tcore(ctx->stream);
  double nu = 0;
  st = fp64 ? nystrom_core<double>(ctx, m, l, Q, Y64, Cm, R, d_pair, d_scalar, Z, ldz, &nu, dist)
            : nystrom_core<float>(ctx, m, l, Q, Y32, Cm, R, d_pair, d_scalar, Z, ldz, &nu, dist);
  if (st) return st;
  ms_core = tcore.stop_ms();
  if (rep) {
    rep->nu = nu;
    rep->ms_sketch = ms_sketch;
    rep->ms_orth = ms_orth;
    rep->ms_core = ms_core;
  }
  return DB200_OK;
}

}  // namespace db200

using namespace db200;

extern "C" {

void db200_barrier_defaults(db200_barrier_params* p) {
  if (!p) return;
  p->t0 = 1.0;
  p->mu = 20.0;
  p->alpha = 0.1;
  p->beta = 0.5;
  p->gap_tol = 1e-6;
  p->newton_tol = 1e-6;
  p->max_outer = 60;
  p->max_newton = 200;
  p->precision = DB200_MIXED;
  p->refine_max = 6;
  p->bias = 0;
}

int db200_potrf(db200_context* ctx, int n, double* A, int lda, int nb) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 0 || !A || lda < n) return fail(ctx, DB200_ERR_INVALID, "potrf: bad arguments");
  if (n == 0) return DB200_OK;
  int* pair = static_cast<int*>(slot_buffer(ctx, SLOT_SPARE, 256));
  if (!pair) return DB200_ERR_NOMEM;
  DB200_CUDA(ctx, cudaMemsetAsync(pair, 0, 2 * sizeof(int), ctx->stream));
  int st = potrf_upper(ctx, A, lda, n, pair, pair + 1, nb <= 0 ? 64 : nb);
  if (st) return st;
  int pst = 0, bad = 0;
  if ((st = read_status(ctx, pair, &pst, &bad))) return st;
  if (pst) return fail(ctx, DB200_ERR_NOT_SPD, "potrf: non-positive pivot in the block starting at row " +
                                                   std::to_string(bad));
  return DB200_OK;
}

int db200_cholqr2(db200_context* ctx, int n, int l, double* Y, int ldy, double* R, int ldr) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < l || l < 1 || !Y || ldy < n || (R && ldr < l)) return fail(ctx, DB200_ERR_INVALID, "cholqr2: bad arguments");
  int st = cholqr2_impl(ctx, n, l, Y, ldy, R, ldr, false);
  if (st) return st;
  return db200_synchronize(ctx);
}

int db200_gemm_tn(db200_context* ctx, int k, int m, int n, double alpha, const double* A, int lda, const double* B,
                  int ldb, double beta, double* C, int ldc) {
  if (!ctx) return DB200_ERR_INVALID;
  if (k < 0 || m < 0 || n < 0 || !A || !B || !C || lda < k || ldb < k || ldc < m)
    return fail(ctx, DB200_ERR_INVALID, "gemm_tn: bad arguments");
  return gram<double, double>(ctx, k, m, n, A, lda, B, ldb, nullptr, alpha, beta, C, ldc, false);
}

int db200_trsm_lutn(db200_context* ctx, int m, int n, const double* R, int ldr, double* B, int ldb) {
  if (!ctx) return DB200_ERR_INVALID;
  if (m < 0 || n < 0 || !R || !B || ldr < m || ldb < m) return fail(ctx, DB200_ERR_INVALID, "trsm: bad arguments");
  if (m == 0 || n == 0) return DB200_OK;
  // B <- (R^-1)^T B:  X = R^-1 (triangular inverse), then B = X^T B through the Gram kernel into scratch
  const size_t bytes = 1024 + align_up((size_t)m * m * 8, 256) + align_up((size_t)m * n * 8, 256);
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_SPARE, bytes));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  double* Xi = cv.take<double>((size_t)m * m);
  double* T = cv.take<double>((size_t)m * n);
  int st = trinv_upper(ctx, R, ldr, m, Xi, m);
  if (!st) st = gram<double, double>(ctx, m, m, n, Xi, m, B, ldb, nullptr, 1.0, 0.0, T, m, false);
  if (st) return st;
  DB200_CUDA(ctx, cudaMemcpy2DAsync(B, sizeof(double) * ldb, T, sizeof(double) * m, sizeof(double) * m, n,
                                    cudaMemcpyDeviceToDevice, ctx->stream));
  return db200_synchronize(ctx);
}

int db200_svm_barrier(db200_context* ctx, int n, int r, const double* Z, int ldz, const float* y, double C,
                      const db200_barrier_params* p, double* a, db200_svm_report* rep) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 1 || r < 1 || !Z || ldz < n || !y || !a || !(C > 0)) return fail(ctx, DB200_ERR_INVALID, "svm_barrier: bad arguments");
  db200_barrier_params P;
  if (p) P = *p;
  else db200_barrier_defaults(&P);
  int st = svm_barrier_impl(ctx, n, r, Z, ldz, y, C, P, a, rep, sharded(ctx));
  if (st && st != DB200_ERR_MAXITER) return st;
  int s2 = db200_synchronize(ctx);
  return s2 ? s2 : st;
}

int db200_lowrank(db200_context* ctx, int n, int d, int l, int q, const float* X, int ldx, const float* y,
                  const float* Omega, int ldo, float gamma, int precision, double* Z, int ldz, db200_svm_report* rep) {
  if (!ctx) return DB200_ERR_INVALID;
  int s0 = 0, rows = n;  // rows of Z this rank writes
  if (sharded(ctx) && n >= 0) db200_row_shard(n, ctx->coll_world, ctx->coll_rank, &s0, &rows);
  if (n < 1 || d < 1 || l < 1 || q < 0 || !X || ldx < d || !y || !Omega || ldo < n || !Z || ldz < rows ||
      (precision != DB200_MIXED && precision != DB200_FP64 && precision != DB200_MIXED_FAST))
    return fail(ctx, DB200_ERR_INVALID, "lowrank: bad arguments");
  int st = lowrank_impl(ctx, n, d, l, q, X, ldx, y, Omega, ldo, gamma, precision, Z, ldz, rep, sharded(ctx));
  if (st) return st;
  return db200_synchronize(ctx);
}

int db200_svm_solve(db200_context* ctx, int n, int d, int l, int q, const float* X, int ldx, const float* y,
                    const float* Omega, int ldo, float gamma, double C, const db200_barrier_params* p, double* a,
                    double* Z, int ldz, db200_svm_report* rep) {
  if (!ctx) return DB200_ERR_INVALID;
  EventTimer total(ctx->stream);
  db200_svm_report local;
  std::memset(&local, 0, sizeof(local));
  db200_barrier_params P;
  if (p) P = *p;
  else db200_barrier_defaults(&P);
  int st = db200_lowrank(ctx, n, d, l, q, X, ldx, y, Omega, ldo, gamma, P.precision, Z, ldz, &local);
  if (st) return st;
  // row-sharded: the barrier runs over this rank's rows of Z, y and a
  int s0 = 0, rows = n;
  if (sharded(ctx)) db200_row_shard(n, ctx->coll_world, ctx->coll_rank, &s0, &rows);
  st = db200_svm_barrier(ctx, rows, l, Z, ldz, y + s0, C, &P, a, &local);
  local.ms_total = total.stop_ms();
  if (rep) *rep = local;
  return st;
}

}  // extern "C"
