// Remaining C ABI: memory helpers for callers that stage host data (the one-rank DArray mirror in
// include/darray_b200/), general FP64/FP32 GEMM, singular values, the Knorm residual, the Woodbury solve and
// the barrier terms of include/dbarrier.h:14-81 on device data, plus the process-wide default context.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "barrier.h"
#include "internal.h"
#include "la64.h"

using namespace db200;

namespace {
std::mutex g_default_mutex;
db200_context* g_default = nullptr;

bool is_n(char c) { return c == 'N' || c == 'n'; }
bool is_t(char c) { return c == 'T' || c == 't' || c == 'C' || c == 'c'; }
}  // namespace

extern "C" {

db200_context* db200_default_context(void) {
  std::lock_guard<std::mutex> lock(g_default_mutex);
  if (!g_default) {
    if (db200_create(&g_default, 0, DB200_OWN_STREAM) != DB200_OK) g_default = nullptr;
  }
  return g_default;
}

int db200_release_default_context(void) {
  std::lock_guard<std::mutex> lock(g_default_mutex);
  int st = db200_destroy(g_default);
  g_default = nullptr;
  return st;
}

int db200_malloc(db200_context* ctx, size_t bytes, void** ptr) {
  if (!ctx || !ptr) return DB200_ERR_INVALID;
  *ptr = nullptr;
  if (bytes == 0) return DB200_OK;
  DB200_CUDA(ctx, cudaMalloc(ptr, bytes));
  return DB200_OK;
}

int db200_free(db200_context* ctx, void* ptr) {
  if (!ctx) return DB200_ERR_INVALID;
  if (!ptr) return DB200_OK;
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  DB200_CUDA(ctx, cudaFree(ptr));
  return DB200_OK;
}

int db200_copy_to_device(db200_context* ctx, void* dst, const void* src, size_t bytes) {
  if (!ctx || (bytes && (!dst || !src))) return DB200_ERR_INVALID;
  if (!bytes) return DB200_OK;
  DB200_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return DB200_OK;
}

int db200_copy_to_host(db200_context* ctx, void* dst, const void* src, size_t bytes) {
  if (!ctx || (bytes && (!dst || !src))) return DB200_ERR_INVALID;
  if (!bytes) return DB200_OK;
  DB200_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  return db200_synchronize(ctx);
}

int db200_gemm(db200_context* ctx, char ta, char tb, int m, int n, int k, double alpha, const double* A, int lda,
               const double* B, int ldb, double beta, double* C, int ldc) {
  if (!ctx) return DB200_ERR_INVALID;
  if (m < 0 || n < 0 || k < 0 || !A || !B || !C || ldc < m) return fail(ctx, DB200_ERR_INVALID, "gemm: bad arguments");
  if (m == 0 || n == 0) return DB200_OK;
  if (is_n(ta) && (is_n(tb) || is_t(tb))) {
    if (lda < m || (is_n(tb) ? ldb < k : ldb < n)) return fail(ctx, DB200_ERR_INVALID, "gemm: bad leading dimension");
    return gemm_tall<double, double>(ctx, m, k, n, A, lda, B, ldb, is_t(tb), beta, C, ldc, alpha);
  }
  if (is_t(ta) && is_n(tb)) {
    if (lda < k || ldb < k) return fail(ctx, DB200_ERR_INVALID, "gemm: bad leading dimension");
    return gram<double, double>(ctx, k, m, n, A, lda, B, ldb, nullptr, alpha, beta, C, ldc, false);
  }
  return fail(ctx, DB200_ERR_UNSUPPORTED, "gemm: op(A) = A^T with op(B) = B^T is not provided");
}

int db200_sgemm(db200_context* ctx, char ta, char tb, int m, int n, int k, float alpha, const float* A, int lda,
                const float* B, int ldb, float beta, float* C, int ldc) {
  if (!ctx) return DB200_ERR_INVALID;
  if (m < 0 || n < 0 || k < 0 || !A || !B || !C || ldc < m) return fail(ctx, DB200_ERR_INVALID, "sgemm: bad arguments");
  if (m == 0 || n == 0) return DB200_OK;
  if (is_n(ta) && is_n(tb)) {
    // C = alpha A B + beta C: B (k x n) widened to FP64 in scratch, FP64 accumulation
    if (lda < m || ldb < k) return fail(ctx, DB200_ERR_INVALID, "sgemm: bad leading dimension");
    double* Bd = static_cast<double*>(slot_buffer(ctx, SLOT_SPARE, (size_t)k * n * 8 + 256));
    if (!Bd) return DB200_ERR_NOMEM;
    int st = convert<float, double>(ctx, B, ldb, Bd, k, k, n);
    if (st) return st;
    return gemm_tall<float, float>(ctx, m, k, n, A, lda, Bd, k, false, beta, C, ldc, alpha);
  }
  if (is_t(ta) && is_n(tb)) {
    if (lda < k || ldb < k) return fail(ctx, DB200_ERR_INVALID, "sgemm: bad leading dimension");
    double* T = static_cast<double*>(slot_buffer(ctx, SLOT_SPARE, (size_t)m * n * 8 + 256));
    if (!T) return DB200_ERR_NOMEM;
    int st = gram<float, float>(ctx, k, m, n, A, lda, B, ldb, nullptr, 1.0, 0.0, T, m, false);
    if (st) return st;
    return axpby_f32(ctx, C, ldc, T, m, m, n, alpha, beta);
  }
  return fail(ctx, DB200_ERR_UNSUPPORTED, "sgemm: only (N,N) and (T,N) are provided, as in tc_sgemm");
}

int db200_svd_values(db200_context* ctx, int n, double* A, int lda, double* S) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 0 || !A || !S || lda < n) return fail(ctx, DB200_ERR_INVALID, "svd_values: bad arguments");
  if (n == 0) return DB200_OK;
  if (n > 8192) return fail(ctx, DB200_ERR_UNSUPPORTED, "svd_values: n > 8192");
  int* d_status = static_cast<int*>(slot_buffer(ctx, SLOT_SPARE, 256));
  if (!d_status) return DB200_ERR_NOMEM;
  int st = jacobi_svd_values(ctx, A, lda, n, S, d_status);
  if (!st) st = sort_desc(ctx, S, n);
  if (st) return st;
  int h = 0;
  DB200_CUDA(ctx, cudaMemcpyAsync(&h, d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (h) return fail(ctx, DB200_ERR_MAXITER, "svd_values: Jacobi sweeps did not converge");
  return DB200_OK;
}

int db200_knorm(db200_context* ctx, int n, int d, int k, const float* X, int ldx, const float* y, const double* Z,
                int ldz, float gamma, double* out3) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 1 || d < 1 || k < 1 || !X || ldx < d || !Z || ldz < n || !out3)
    return fail(ctx, DB200_ERR_INVALID, "knorm: bad arguments");
  const int b = n < 2048 ? n : 2048;  // row block of K held in fp32
  const size_t bytes = 256 + align_up((size_t)b * n * 4, 256) + 256;
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_PIPE, bytes));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  double* sums = cv.take<double>(4);
  float* Kb = cv.take<float>((size_t)b * n);
  DB200_CUDA(ctx, cudaMemsetAsync(sums, 0, 4 * sizeof(double), ctx->stream));
  int st;
  for (int i0 = 0; i0 < n; i0 += b) {
    const int rb = (n - i0 < b) ? n - i0 : b;
    if ((st = db200_rbf_block(ctx, rb, n, d, X + (size_t)i0 * ldx, ldx, X, ldx, DB200_POINT_MAJOR,
                              y ? y + i0 : nullptr, y, Kb, rb, gamma)))
      return st;
    if ((st = sumsq_f32(ctx, Kb, rb, rb, n, sums))) return st;
    // Kb <- Z_i Z^T - Kb  (FP64 accumulation)
    if ((st = gemm_tall<double, float>(ctx, rb, k, n, Z + i0, ldz, Z, ldz, true, -1.0, Kb, rb, 1.0))) return st;
    if ((st = sumsq_f32(ctx, Kb, rb, rb, n, sums + 1))) return st;
  }
  double h[2];
  DB200_CUDA(ctx, cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  st = db200_synchronize(ctx);
  if (st) return st;
  out3[0] = std::sqrt(h[0]);
  out3[1] = std::sqrt(h[1]);
  out3[2] = h[0] > 0 ? std::sqrt(h[1] / h[0]) : 0.0;
  return DB200_OK;
}

int db200_woodbury_solve(db200_context* ctx, int n, int r, const double* Z, int ldz, const double* diag,
                         const double* b, double* x) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 1 || r < 1 || r > 4096 || !Z || ldz < n || !diag || !b || !x)
    return fail(ctx, DB200_ERR_INVALID, "woodbury_solve: bad arguments");
  // (Z Z^T + diag(g))^-1 b = g^-1 b - g^-1 Z (I + Z^T g^-1 Z)^-1 Z^T g^-1 b
  const size_t rr = (size_t)r * r;
  const size_t bytes = 1024 + 2 * align_up((size_t)n * 8, 256) + 2 * align_up(rr * 8, 256) + align_up((size_t)r * 8, 256);
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_SPARE, bytes));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  int* pair = cv.take<int>(4);
  double* red = cv.take<double>(8);
  double* ginv = cv.take<double>(n);
  double* nb = cv.take<double>(n);
  double* M = cv.take<double>(rr);
  double* L = cv.take<double>(rr);
  double* u = cv.take<double>(r);
  int st = bar_reciprocal(ctx, n, diag, ginv);
  if (!st) st = gram<double, double>(ctx, n, r, r, Z, ldz, Z, ldz, ginv, 1.0, 0.0, M, r, true);
  if (!st) st = bar_add_identity(ctx, M, r, r);
  if (!st) st = bar_gemv_t(ctx, n, r, Z, ldz, b, ginv, 1.0, u);  // u = Z^T g^-1 b, solved below for M^-1 Z^T g^-1 b
  if (st) return st;
  DB200_CUDA(ctx, cudaMemsetAsync(pair, 0, 2 * sizeof(int), ctx->stream));
  if ((st = potrf_upper(ctx, M, r, r, pair, pair + 1))) return st;
  if ((st = transpose64(ctx, M, r, r, r, L, r))) return st;
  if ((st = trsv_upper(ctx, M, L, r, r, u, true))) return st;
  if ((st = trsv_upper(ctx, M, L, r, r, u, false))) return st;
  // u = M^-1 Z^T g^-1 b now; x = g^-1 (b - Z u) is the direction kernel's -dinv (h + Z u) with h = -b
  if ((st = bar_negate(ctx, n, b, nb))) return st;
  if ((st = bar_init_red(ctx, red, 2, 0, 1))) return st;
  if ((st = bar_direction(ctx, n, r, Z, ldz, u, nb, ginv, ginv, 1e300, x, red))) return st;
  int h[2] = {0, 0};
  DB200_CUDA(ctx, cudaMemcpyAsync(h, pair, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  st = db200_synchronize(ctx);
  if (st) return st;
  if (h[0]) return fail(ctx, DB200_ERR_NOT_SPD, "woodbury_solve: capacity matrix not positive definite");
  return DB200_OK;
}

int db200_gram_weighted(db200_context* ctx, int n, int r, const double* Z, int ldz, const double* w, double* M, int ldm,
                        int use_tensor_cores) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 1 || r < 1 || !Z || ldz < n || !M || ldm < r) return fail(ctx, DB200_ERR_INVALID, "gram_weighted: bad arguments");
  if (!use_tensor_cores) return gram<double, double>(ctx, n, r, r, Z, ldz, Z, ldz, w, 1.0, 0.0, M, ldm, true);
  void* scratch = slot_buffer(ctx, SLOT_SPARE, gram_tc_scratch_bytes(n, r));
  if (!scratch) return DB200_ERR_NOMEM;
  DB200_CUDA(ctx, cudaMemset2DAsync(M, sizeof(double) * ldm, 0, sizeof(double) * r, r, ctx->stream));
  return gram_tc_weighted(ctx, n, r, Z, ldz, w, M, ldm, scratch, use_tensor_cores >= 5 ? use_tensor_cores : 8);
}

int db200_rbf_sketch_f64(db200_context* ctx, int m, int n, int d, int l, const float* Xi, int ldxi, const float* Xj,
                         int ldxj, const float* yi, const float* yj, const double* Omega, int ldo, double* Y, int ldy,
                         double gamma) {
  if (!ctx) return DB200_ERR_INVALID;
  if (m < 0 || n < 0 || d < 1 || l < 0 || !Xi || !Xj || ldxi < d || ldxj < d || !Omega || ldo < n || !Y || ldy < m)
    return fail(ctx, DB200_ERR_INVALID, "rbf_sketch_f64: bad arguments");
  if (m == 0 || l == 0) return DB200_OK;
  if (n == 0) {
    DB200_CUDA(ctx, cudaMemset2DAsync(Y, sizeof(double) * (size_t)ldy, 0, sizeof(double) * (size_t)m, (size_t)l,
                                      ctx->stream));
    return DB200_OK;
  }
  if (d > 256) return fail(ctx, DB200_ERR_UNSUPPORTED, "rbf_sketch_f64: d > 256 not supported");
  // one fused launch: FP64 DMMA distances, FP64 exp, FP64 DMMA sketch product; K never leaves the SM
  return rbf_sketch_f64_fused(ctx, m, n, d, l, Xi, ldxi, Xj, ldxj, yi, yj, Omega, ldo, Y, ldy, gamma);
}

int db200_rbf_block_f64(db200_context* ctx, int m, int n, int d, const float* Xi, int ldxi, const float* Xj,
                        int ldxj, const float* yi, const float* yj, double* K, int ldk, double gamma) {
  if (!ctx) return DB200_ERR_INVALID;
  if (m < 0 || n < 0 || d < 1 || !Xi || !Xj || ldxi < d || ldxj < d || !K || ldk < m)
    return fail(ctx, DB200_ERR_INVALID, "rbf_block_f64: bad arguments");
  if (m == 0 || n == 0) return DB200_OK;
  const size_t bytes = 1024 + align_up((size_t)(m + n) * 8, 256) + 1024;
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_SPARE, bytes));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  double* si = cv.take<double>(m);
  double* sj = cv.take<double>(n);
  int st = rownorm_f64(ctx, Xi, ldxi, m, d, si);
  if (!st) st = rownorm_f64(ctx, Xj, ldxj, n, d, sj);
  // G = Xi Xj^T on the FP64 tensor cores (the Gram kernel over the d features), then K in place
  if (!st) st = gram<float, float>(ctx, d, m, n, Xi, ldxi, Xj, ldxj, nullptr, 1.0, 0.0, K, ldk, false);
  if (!st) st = rbf_from_gram_f64(ctx, K, ldk, m, n, si, sj, yi, yj, gamma);
  return st;
}

int db200_vec_update(db200_context* ctx, int n, double alpha, const double* x, double beta, double* y,
                      double gamma) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 0 || !y) return fail(ctx, DB200_ERR_INVALID, "vec_update: bad arguments");
  if (n == 0) return DB200_OK;
  return bar_vec_update(ctx, n, alpha, x, beta, y, gamma);
}

int db200_barrier_terms(db200_context* ctx, int n, int k, const double* Z, int ldz, const double* a, double C,
                        double t, double* gradf, double* gradphi, double* grad, double* D, double* f_gg) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 1 || k < 1 || k > 4096 || !Z || ldz < n || !a || !f_gg)
    return fail(ctx, DB200_ERR_INVALID, "barrier_terms: bad arguments");
  const size_t bytes = 1024 + 4 * align_up((size_t)n * 8, 256) + align_up((size_t)k * 8, 256);
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_SPARE, bytes));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  double* red = cv.take<double>(16);
  double* w = cv.take<double>(k);
  double* gf = cv.take<double>(n);
  double* gp = cv.take<double>(n);
  double* g = cv.take<double>(n);
  double* dd = cv.take<double>(n);
  int st = bar_gemv_t(ctx, n, k, Z, ldz, a, nullptr, 1.0, w);
  if (!st) st = bar_init_red(ctx, red, 2, 1, 1);
  if (!st) st = bar_terms(ctx, n, k, Z, ldz, w, a, C, t, gf, gp, g, dd, red);
  if (!st) st = bar_dot(ctx, k, w, w, red + 8);
  if (st) return st;
  double h[9];
  DB200_CUDA(ctx, cudaMemcpyAsync(h, red, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  if ((st = db200_synchronize(ctx))) return st;
  const double f = 0.5 * h[8] - h[0];
  f_gg[0] = f;
  f_gg[1] = f - h[1] / t;
  auto out = [&](double* dst, const double* src) -> int {
    if (dst) DB200_CUDA(ctx, cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    return DB200_OK;
  };
  if ((st = out(gradf, gf)) || (st = out(gradphi, gp)) || (st = out(grad, g)) || (st = out(D, dd))) return st;
  return db200_synchronize(ctx);
}

}  // extern "C"
