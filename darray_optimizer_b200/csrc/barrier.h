// Device building blocks of the barrier solver (barrier.cu); FP64, column-major Z (n x r, leading dim ld).
#pragma once
#include "internal.h"

namespace db200 {

// red[0..nsum) = 0, next nmax = 0 (for maxima of non-negative values), next nmin = DBL_MAX.
int bar_init_red(db200_context* ctx, double* red, int nsum, int nmax, int nmin);
// g = Z w - 1 + (-1/a + 1/(C-a))/t,  dinv = 1/D,  D = (1/a^2 + 1/(C-a)^2)/t  (include/dbarrier.h:48-81);
// red: [0] += sum a, [1] += sum(log a + log(C-a)), [2] max D, [3] min D.  zw_in: Z w given (no pass over Z);
// zw_out: Z w stored.
int bar_grad_hess(db200_context* ctx, int n, int r, const double* Z, long long ld, const double* w, const double* a,
                  double C, double t, double* g, double* dinv, double* red, const double* zw_in = nullptr,
                  double* zw_out = nullptr);
// s = -dinv (g + Z u);  red: [0] += g.s, [1] += sum s, [2] min feasible step (init DBL_MAX).
int bar_direction(db200_context* ctx, int n, int r, const double* Z, long long ld, const double* u, const double* g,
                  const double* dinv, const double* a, double C, double* s, double* red);
// out = sign * Z^T (scale .* v)  (scale may be null); out is zeroed first.
int bar_gemv_t(db200_context* ctx, int n, int r, const double* Z, long long ld, const double* v, const double* scale,
               double sign, double* out);
// out[k] = sum log(a + tau_k s) + log(C - a - tau_k s), out[16 + k] = count of coordinates leaving the box.
int bar_linesearch16(db200_context* ctx, int n, const double* a, const double* s, double C, const double* taus,
                     double* out);
int bar_axpy(db200_context* ctx, int n, double alpha, const double* x, double* y);
// gradf, gradphi, grad, D of include/dbarrier.h:48-81 separately; red: [0] += sum a, [1] += sum logs.
int bar_terms(db200_context* ctx, int n, int r, const double* Z, long long ld, const double* w, const double* a,
              double C, double t, double* gf, double* gp, double* g, double* D, double* red);
int bar_reciprocal(db200_context* ctx, int n, const double* x, double* y);
// res = g + Z v + s/dinv (v = Z^T s: the negated Newton residual); red [0] += |res|^2, [1] += |g|^2; zv_out: Z v
// stored
int bar_residual(db200_context* ctx, int n, int r, const double* Z, long long ld, const double* v, const double* g,
                 const double* dinv, const double* s, double* res, double* red, double* zv_out = nullptr);
// red [0] += g.s, [1] += sum s, [2] min feasible step (init DBL_MAX)
int bar_step_stats(db200_context* ctx, int n, const double* g, const double* s, const double* a, double C,
                   double* red);

// gram_tc.cu: M (upper, FP64) += (D^-1/2 Z)^T (D^-1/2 Z) on the int8 tensor cores (Ozaki slices)
size_t gram_tc_scratch_bytes(int n, int r);
int gram_tc_weighted(db200_context* ctx, int n, int r, const double* Z, long long ldz, const double* w, double* M,
                     int ldm, void* scratch, int slices = 8);
int bar_negate(db200_context* ctx, int n, const double* x, double* y);
// y = alpha x + beta y + gamma (x may be null)
int bar_vec_update(db200_context* ctx, int n, double alpha, const double* x, double beta, double* y, double gamma);
// red[0] = sum max(0, 1 - (Z w)_i - y_i b)  (y null: no bias term)
int bar_hinge(db200_context* ctx, int n, int r, const double* Z, long long ld, const double* w, double* red,
              const double* y = nullptr, double b = 0.0);
int bar_add_identity(db200_context* ctx, double* M, int ldm, int r);
int bar_scale_diag(db200_context* ctx, double* M, int ldm, int r, double factor);
int bar_dot(db200_context* ctx, int r, const double* x, const double* y, double* out);
// taus[k] = min(1, 0.99 * *step_max) beta^k for k < 16 (the line search's first candidates, formed on the device)
int bar_steps16(db200_context* ctx, const double* step_max, double beta, double* taus);

}  // namespace db200
