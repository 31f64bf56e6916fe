// One-rank mirror of include/blas_like.h: matrix_multiply (T,N) and triangular_solve (L,U,T) on the GPU.
#pragma once
#include <cassert>
#include <vector>
#include "cblas_like.h"
#include "darray.h"
#include "detail.h"

namespace DArray {

// C = alpha A^T B + beta C on descriptor blocks (include/blas_like.h:63-93; only ("T","N"), as in the reference).
template <typename T>
void matrix_multiply(const char* transa, const char* transb, DMatrixDescriptor<T> Adesc, DMatrixDescriptor<T> Bdesc,
                     DMatrixDescriptor<T> Cdesc, T alpha, T beta, int bs = 128) {
  (void)bs;
  using namespace darray_b200::detail;
  if (!((*transa == 'T' || *transa == 't') && (*transb == 'N' || *transb == 'n'))) {
    assert(0 && "matrix_multiply: only (T, N) is provided, as in the reference");
    return;
  }
  const int k = Adesc.m(), m = Adesc.n(), n = Bdesc.n();
  assert(Bdesc.m() == k && Cdesc.m() == m && Cdesc.n() == n);
  T* A = Adesc.matrix.data() + Adesc.i1 + (size_t)Adesc.j1 * Adesc.matrix.lld();
  T* B = Bdesc.matrix.data() + Bdesc.i1 + (size_t)Bdesc.j1 * Bdesc.matrix.lld();
  T* C = Cdesc.matrix.data() + Cdesc.i1 + (size_t)Cdesc.j1 * Cdesc.matrix.lld();
  Dev<double> da((size_t)k * m), db((size_t)k * n), dc((size_t)m * n);
  upload(da, A, k, m, Adesc.matrix.lld());
  upload(db, B, k, n, Bdesc.matrix.lld());
  upload(dc, C, m, n, Cdesc.matrix.lld());
  check(db200_gemm(ctx(), 'T', 'N', m, n, k, (double)alpha, da.p, k, db.p, k, (double)beta, dc.p, m), "matrix_multiply");
  download(C, m, n, Cdesc.matrix.lld(), dc);
}

// B <- U^-T B with U the upper triangle of the m x m block A (include/blas_like.h:96-127; only ("L","U","T"),
// non-unit diagonal).  Like the reference, alpha is not applied.
template <typename T>
void triangular_solve(const char* side, const char* uplo, const char* transa, const char* diag, int m, int n, T alpha,
                      DMatrixDescriptor<T> Adesc, DMatrixDescriptor<T> Bdesc, int bs = 64) {
  (void)alpha;
  (void)bs;
  using namespace darray_b200::detail;
  if (!((*side == 'L' || *side == 'l') && (*uplo == 'U' || *uplo == 'u') && (*transa == 'T' || *transa == 't') &&
        (*diag == 'N' || *diag == 'n'))) {
    assert(0 && "triangular_solve: only (L, U, T, N) is provided, as in the reference");
    return;
  }
  T* A = Adesc.matrix.data() + Adesc.i1 + (size_t)Adesc.j1 * Adesc.matrix.lld();
  T* B = Bdesc.matrix.data() + Bdesc.i1 + (size_t)Bdesc.j1 * Bdesc.matrix.lld();
  Dev<double> da((size_t)m * m), db((size_t)m * n);
  upload(da, A, m, m, Adesc.matrix.lld());
  upload(db, B, m, n, Bdesc.matrix.lld());
  check(db200_trsm_lutn(ctx(), m, n, da.p, m, db.p, m), "triangular_solve");
  download(B, m, n, Bdesc.matrix.lld(), db);
}

// C = alpha L U + beta C with L the unit lower triangle of A and U the upper triangle of B, all n x n
// (include/blas_like.h:9-60: the product that checks an LU factorisation).  FP64 product on the GPU.
template <typename T>
void triangular_triangular_multiply(DMatrix<T>& A, DMatrix<T>& B, DMatrix<T>& C, T alpha, T beta) {
  using namespace darray_b200::detail;
  const int n = C.dims()[0];
  assert(C.dims()[1] == n && A.dims()[0] == n && B.dims()[1] == n);
  std::vector<double> L((size_t)n * n, 0.0), U((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      if (i > j) L[i + (size_t)j * n] = A(i, j);
      else if (i == j) L[i + (size_t)j * n] = 1.0;
      if (i <= j) U[i + (size_t)j * n] = B(i, j);
    }
  Dev<double> dl((size_t)n * n), du((size_t)n * n), dc((size_t)n * n);
  upload(dl, L.data(), n, n, n);
  upload(du, U.data(), n, n, n);
  upload(dc, C.data(), n, n, C.lld());
  check(db200_gemm(ctx(), 'N', 'N', n, n, n, (double)alpha, dl.p, n, du.p, n, (double)beta, dc.p, n),
        "triangular_triangular_multiply");
  download(C.data(), n, n, C.lld(), dc);
}

}  // namespace DArray
