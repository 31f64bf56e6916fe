// Driver that exposes the reference's own C++ templates (compiled from the reference sources, at one MPI
// rank) through extern "C" entry points, so that tests/golden/gen_reference_goldens.py can pin the FP64
// oracle against the reference's arithmetic.  Test infrastructure only: built by oracle/build_ref.sh into
// oracle/_ref/, never linked into the product.
#include <cstring>
#include <string>

#include "darray.h"
#include "lapack_like.h"
#include "blas_like.h"
#include "dbarrier.h"
#include "read_input.h"

using DArray::DMatrix;
using DArray::DMatrixDescriptor;
using DArray::Grid;
using DArray::LMatrix;

namespace {
Grid& grid() {
  static Grid g(MPI_COMM_WORLD, 1, 1);
  return g;
}
void load(DMatrix<float>& M, const float* src, int m, int n) {
  for (int j = 0; j < n; ++j) std::memcpy(M.data() + (size_t)j * M.lld(), src + (size_t)j * m, sizeof(float) * m);
}
void store(DMatrix<float>& M, float* dst, int m, int n) {
  for (int j = 0; j < n; ++j) std::memcpy(dst + (size_t)j * m, M.data() + (size_t)j * M.lld(), sizeof(float) * m);
}
LMatrix<double> lmat(double* p, int m, int n) { return LMatrix<double>(m, n, m, p); }
}  // namespace

extern "C" {

// cholesky_factorize / cholesky_factorize_recursive (include/lapack_like.h:10,59): A (n x n, column major) is
// overwritten; only the upper triangle is meaningful on return.
void ref_cholesky(float* A, int n, int bs, int recursive) {
  DMatrix<float> M(grid(), n, n);
  load(M, A, n, n);
  if (recursive)
    DArray::cholesky_factorize_recursive(M, 'U', n, 0, bs);
  else
    DArray::cholesky_factorize(M, 'U', n, 0, bs);
  store(M, A, n, n);
}

// tall_skinny_qr_factorize (include/lapack_like.h:283): A (m x n) is overwritten by Q; R (n x n) returned.
void ref_tsqr(float* A, int m, int n, float* R) {
  DMatrix<float> M(grid(), m, n);
  load(M, A, m, n);
  auto Rl = DArray::tall_skinny_qr_factorize(M, 0, 0, m, n);
  store(M, A, m, n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) R[i + j * n] = Rl.data()[i + j * Rl.ld()];
}

// svd (include/lapack_like.h:389): singular values of the n x n matrix A.
void ref_svd(float* A, int n, float* S) {
  LMatrix<float> L(n, n);
  std::memcpy(L.data(), A, sizeof(float) * n * n);
  auto s = DArray::svd<float>(0, L, 0, 0, n, n);
  std::memcpy(S, s.data(), sizeof(float) * n);
}

// triangular_solve("L","U","T","N") (include/blas_like.h:96): B(m x n) <- U^-T B, U is the upper triangle of A.
void ref_triangular_solve(const float* A, float* B, int m, int n, int bs) {
  DMatrix<float> MA(grid(), m, m), MB(grid(), m, n);
  load(MA, A, m, m);
  load(MB, B, m, n);
  DMatrixDescriptor<float> Ad{MA, 0, 0, m, m}, Bd{MB, 0, 0, m, n};
  DArray::triangular_solve("L", "U", "T", "N", m, n, 1.0f, Ad, Bd, bs);
  store(MB, B, m, n);
}

// matrix_multiply("T","N") (include/blas_like.h:63): C(m x n) <- alpha A^T B + beta C, A is k x m, B is k x n.
void ref_matrix_multiply_tn(const float* A, const float* B, float* C, int k, int m, int n, float alpha, float beta,
                            int bs) {
  DMatrix<float> MA(grid(), k, m), MB(grid(), k, n), MC(grid(), m, n);
  load(MA, A, k, m);
  load(MB, B, k, n);
  load(MC, C, m, n);
  DMatrixDescriptor<float> Ad{MA, 0, 0, k, m}, Bd{MB, 0, 0, k, n}, Cd{MC, 0, 0, m, n};
  DArray::matrix_multiply("T", "N", Ad, Bd, Cd, alpha, beta, bs);
  store(MC, C, m, n);
}

// include/dbarrier.h:14-81 on caller-owned FP64 buffers (Z n x k column major).
double ref_f(int n, int k, double* a, double* Z) {
  auto A = lmat(a, n, 1);
  auto M = lmat(Z, n, k);
  return DArray::f<double>(0, n, k, A, M);
}
double ref_gg(int n, int k, double* a, double* Z, double C, double t) {
  auto A = lmat(a, n, 1);
  auto M = lmat(Z, n, k);
  return DArray::gg<double>(0, n, k, A, M, C, t);
}
void ref_grad_f(int n, int k, double* Z, double* a, double* out) {
  auto M = lmat(Z, n, k);
  auto A = lmat(a, n, 1);
  auto G = lmat(out, n, 1);
  DArray::Grad_f<double>(n, k, M, A, G);
}
void ref_grad_phi(int n, double* a, double C, double t, double* out) {
  auto A = lmat(a, n, 1);
  auto G = lmat(out, n, 1);
  DArray::Grad_Phi<double>(n, A, C, t, G);
}
void ref_grad(int n, double* gf, double* gp, double* out) {
  auto A = lmat(gf, n, 1), B = lmat(gp, n, 1), G = lmat(out, n, 1);
  DArray::Grad<double>(n, A, B, G);
}
void ref_hess_phi(int n, double* a, double C, double t, double* out) {
  auto A = lmat(a, n, 1);
  auto D = lmat(out, n, 1);
  DArray::Hess_Phi<double>(n, A, C, t, D);
}
// pre_conjgrad (include/dbarrier.h:84-139): x returned in `out`.
void ref_pre_conjgrad(int n, int k, double* Z, double* M, double* D, double* b, double* a, double* out) {
  auto Zm = lmat(Z, n, k), Mm = lmat(M, n, 1), Dm = lmat(D, n, 1), bm = lmat(b, n, 1), am = lmat(a, n, 1);
  auto x = DArray::pre_conjgrad<double>(1, n, k, Zm, Mm, Dm, bm, am);
  std::memcpy(out, x.data(), sizeof(double) * n);
}
// writemodel (include/dbarrier.h:395): X is d x n column major (point-major), Y n labels.
void ref_writemodel(const char* path, int n, int d, int k, double* a, double C, double* Z, double* Y, double* X,
                    double gamma, int minus, int plus) {
  auto A = lmat(a, n, 1), Zm = lmat(Z, n, k), Ym = lmat(Y, n, 1);
  LMatrix<double> Xm(d, n, d, X);
  DArray::writemodel<double>(std::string(path), n, d, k, A, C, Zm, Ym, Xm, gamma, minus, plus);
}
// lu_factorize_partial_pivot (include/lapack_like.h:179-219) on an m x n FP32 matrix (column major, in place)
// with outer block bs; ipiv receives A.ipiv() (1-based global rows).  (The replicate_panel variant, :134-177,
// does not compile when instantiated: :152 passes a std::vector<int> where permute_rows_ipiv takes int*.)
void ref_lu(float* A, int m, int n, int bs, int* ipiv) {
  DMatrix<float> M(grid(), m, n);
  load(M, A, m, n);
  DArray::lu_factorize_partial_pivot(M, 0, 0, m, n, bs);
  store(M, A, m, n);
  const int mn = m < n ? m : n;
  for (int i = 0; i < mn; ++i) ipiv[i] = M.ipiv()[i];
}
// read_input_file<T> (include/read_input.h:8-36): X is d x n column major (point-major), Y n labels.  The
// reference indexes X with stride d and ignores ldx.
void ref_read_input_file_f32(const char* filename, int n, int d, float* X, float* Y) {
  read_input_file<float>(const_cast<char*>(filename), n, d, X, d, Y);
}
void ref_read_input_file_f64(const char* filename, int n, int d, double* X, double* Y) {
  read_input_file<double>(const_cast<char*>(filename), n, d, X, d, Y);
}

}  // extern "C"
