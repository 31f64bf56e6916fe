// One-rank mirror of include/dbarrier.h (low-rank barrier functions, FP64 LMatrix arguments) on the GPU.
// The whole barrier solve is db200_svm_barrier; these per-call functions keep the reference's entry points.
#pragma once
#include <cassert>
#include <cmath>
#include <string>
#include <vector>

#include "darray.h"
#include "detail.h"

namespace DArray {
namespace barrier_detail {
using namespace darray_b200::detail;

// f, gg, gradients and D at x for Z (n x k); any output pointer may be null.
inline void terms(int n, int k, LMatrix<double>& x, LMatrix<double>* Z, double C, double t, double* gradf,
                  double* gradphi, double* grad, double* D, double* f_gg) {
  Dev<double> dz((size_t)n * (k > 0 ? k : 1)), da(n), o1(n), o2(n), o3(n), o4(n);
  if (Z)
    upload(dz, Z->data(), n, k, Z->ld());
  else
    check(db200_vec_update(ctx(), n, 0.0, nullptr, 0.0, dz.p, 0.0), "zero");  // no Z: Z = 0 (n x 1)
  upload(da, x.data(), n, 1, n);
  double fg[2];
  check(db200_barrier_terms(ctx(), n, Z ? k : 1, dz.p, n, da.p, C, t, o1.p, o2.p, o3.p, o4.p, fg), "barrier terms");
  if (gradf) download(gradf, n, 1, n, o1);
  if (gradphi) download(gradphi, n, 1, n, o2);
  if (grad) download(grad, n, 1, n, o3);
  if (D) download(D, n, 1, n, o4);
  if (f_gg) {
    f_gg[0] = fg[0];
    f_gg[1] = fg[1];
  }
}
}  // namespace barrier_detail

// f(x) = 0.5 x^T Z Z^T x - 1^T x (include/dbarrier.h:14-35)
template <typename T>
T f(int rk, int n, int k, LMatrix<T>& x, LMatrix<T>& Z) {
  (void)rk;
  double fg[2];
  barrier_detail::terms(n, k, x, &Z, 1e300, 1.0, nullptr, nullptr, nullptr, nullptr, fg);
  return (T)fg[0];
}

// gg(x) = f(x) - (1/t) sum(log x + log(C - x)) (include/dbarrier.h:38-45)
template <typename T>
T gg(int rk, int n, int k, LMatrix<T>& x, LMatrix<T>& Z, T C, T t) {
  (void)rk;
  double fg[2];
  barrier_detail::terms(n, k, x, &Z, C, t, nullptr, nullptr, nullptr, nullptr, fg);
  return (T)fg[1];
}

// gradf = Z Z^T a - 1 (include/dbarrier.h:48-57)
template <typename T>
void Grad_f(int n, int k, LMatrix<T>& Z, LMatrix<T>& a, LMatrix<T>& gradf) {
  barrier_detail::terms(n, k, a, &Z, 1e300, 1.0, gradf.data(), nullptr, nullptr, nullptr, nullptr);
}

// gradphi = (-1/a + 1/(C - a))/t (include/dbarrier.h:60-65)
template <typename T>
void Grad_Phi(int n, LMatrix<T>& a, T C, T t, LMatrix<T>& gradphi) {
  barrier_detail::terms(n, 0, a, nullptr, C, t, nullptr, gradphi.data(), nullptr, nullptr, nullptr);
}

// grad = gradf + gradphi (include/dbarrier.h:68-73)
template <typename T>
void Grad(int n, LMatrix<T>& gradf, LMatrix<T>& gradphi, LMatrix<T>& grad) {
  using namespace darray_b200::detail;
  Dev<double> x(n), y(n);
  upload(x, gradf.data(), n, 1, n);
  upload(y, gradphi.data(), n, 1, n);
  check(db200_vec_update(ctx(), n, 1.0, x.p, 1.0, y.p, 0.0), "Grad");
  download(grad.data(), n, 1, n, y);
}

// D = (1/a^2 + 1/(C - a)^2)/t (include/dbarrier.h:76-81)
template <typename T>
void Hess_Phi(int n, LMatrix<T>& a, T C, T t, LMatrix<T>& D) {
  barrier_detail::terms(n, 0, a, nullptr, C, t, nullptr, nullptr, nullptr, D.data(), nullptr);
}

// Solution of (Z Z^T + diag(D) + n I) x = b, the system include/dbarrier.h:84-139 iterates on with Jacobi-PCG to
// ||r|| <= 1e-2 from x = a; here solved directly by Sherman-Morrison-Woodbury in FP64 (M and a are not needed).
template <typename T>
LMatrix<T> pre_conjgrad(int rk, int n, int k, LMatrix<T>& Z, LMatrix<T>& M, LMatrix<T>& D, LMatrix<T>& b,
                        LMatrix<T>& a) {
  (void)rk;
  (void)M;
  (void)a;
  using namespace darray_b200::detail;
  Dev<double> dz((size_t)n * k), dd(n), db(n), dx(n);
  upload(dz, Z.data(), n, k, Z.ld());
  upload(dd, D.data(), n, 1, n);
  upload(db, b.data(), n, 1, n);
  check(db200_vec_update(ctx(), n, 0.0, nullptr, 1.0, dd.p, (double)n), "pre_conjgrad shift");
  check(db200_woodbury_solve(ctx(), n, k, dz.p, n, dd.p, db.p, dx.p), "pre_conjgrad");
  LMatrix<T> x(n, 1);
  download(x.data(), n, 1, n, dx);
  return x;
}

// LIBSVM model text with the reference's bias estimate and layout (include/dbarrier.h:395-470).  Host I/O, as
// in the reference; dX is d x n (point-major).  With `bias` (the solve's b, db200_svm_report.b of a solve with
// db200_barrier_params.bias = 1) the model's rho is -b and the reference's estimate from the margin support
// vectors is not made; without it (NULL, the reference's call) the estimate is written.
template <typename T>
void writemodel(const std::string filepath, int n, int d, int k, LMatrix<T>& a, T C, LMatrix<T>& dZ, LMatrix<T> dY,
                LMatrix<T> dX, T gamma, int minus, int plus, const double* bias = nullptr) {
  std::vector<int> sv, bsv;
  for (int i = 0; i < n; ++i)
    if (a.data()[i] > 1e-6) {
      sv.push_back(i);
      if (a.data()[i] < C - 1e-6) bsv.push_back(i);
    }
  std::printf("#BSV %d, #SV %d\n", (int)bsv.size(), (int)sv.size());
  const int nb = bias ? 0 : std::min((int)bsv.size(), 50);
  std::vector<double> bs(nb, 0.0);
  double acc = 0.0;
  for (int j = 0; j < nb; ++j) {
    const int jj = bsv[j];
    double yj = dY[jj];
    for (int ii : sv) {
      double s = 0.0;
      for (int kk = 0; kk < k; ++kk) s += dZ[ii + kk * dZ.ld()] * dZ[ii + kk * dZ.ld()];
      yj -= a[ii] * dY[jj] * s;
    }
    acc += yj;
    bs[j] = yj;
  }
  const double b = bias ? *bias : (nb ? acc / nb : 0.0);
  double sumsq = 0.0;
  for (double v : bs) sumsq += (v - b) * (v - b);
  if (bias) std::printf("b=%.6e from the solve\n ", b);
  else std::printf("approx mean b=%.6e std b=%.6e, #samples=%d\n ", b, nb ? std::sqrt(sumsq / nb) : 0.0, nb);
  FILE* fp = std::fopen(filepath.c_str(), "w");
  if (!fp) return;
  std::fprintf(fp, "svm_type c_svc\n");
  std::fprintf(fp, "kernel_type rbf\n");
  std::fprintf(fp, "gamma %.7f\n", (double)gamma);
  std::fprintf(fp, "nr_class 2\n");
  std::fprintf(fp, "total_sv %d\n", (int)sv.size());
  std::fprintf(fp, "rho %f\n", -b);
  std::fprintf(fp, "label %d %d\n", plus, minus);
  std::fprintf(fp, "nr_sv %d %d\n", (int)bsv.size(), (int)(sv.size() - bsv.size()));
  std::fprintf(fp, "SV\n");
  for (int j : sv) {
    std::fprintf(fp, "%7f ", dY[j] * a[j]);
    for (int kk = 0; kk < d; ++kk) {
      const double v = dX[j * dX.ld() + kk];
      if (v > 0 || v < 0) std::fprintf(fp, "%d:%7f ", kk + 1, dX[j * d + kk]);
    }
    std::fprintf(fp, "\n");
  }
  std::fclose(fp);
}

}  // namespace DArray
