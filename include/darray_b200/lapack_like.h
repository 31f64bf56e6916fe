// One-rank mirror of include/lapack_like.h on the GPU: cholesky_factorize, cholesky_factorize_recursive,
// tall_skinny_qr_factorize and svd (FP64 arithmetic on float or double DMatrix data).  The LU factorisations of
// the reference are not on the kernel-SVM path and are not provided.
#pragma once
#include <algorithm>

#include "blas_like.h"
#include "cblas_like.h"
#include "darray.h"
#include "detail.h"

namespace DArray {

// Upper Cholesky of the n x n block at (gi, gi) in place; only the upper triangle is read and written, as the
// reference's spotrf/strsm/ssyrk('U') sequence does (include/lapack_like.h:10-56).  On a non-positive pivot the
// reference prints and returns; so does this.
template <typename T>
void cholesky_factorize(DMatrix<T>& A, char uplo, int n, int gi, int bs = 256) {
  using namespace darray_b200::detail;
  if (!(uplo == 'U' || uplo == 'u')) {
    assert(0 && "cholesky_factorize: only 'U' is provided, as in the reference");
    return;
  }
  T* a = A.data() + gi + (size_t)gi * A.lld();
  Dev<double> d((size_t)n * n);
  upload(d, a, n, n, A.lld());
  int st = db200_potrf(ctx(), n, d.p, n, std::min(bs, 64));
  if (st == DB200_ERR_NOT_SPD) {
    std::printf("potrf error: %s. Stopping\n", db200_last_error(ctx()));
    return;
  }
  check(st, "cholesky_factorize");
  download(a, n, n, A.lld(), d, true);
}

// Same factor through the recursive formulation's entry point (include/lapack_like.h:59-90).
template <typename T>
void cholesky_factorize_recursive(DMatrix<T>& A, char uplo, int n, int i, int bs = 32) {
  cholesky_factorize(A, uplo, n, i, bs);
}

// Q R of the tall-skinny block A[i1:i2, j1:j2]: Q overwrites the block, R (n x n, upper) is returned
// (include/lapack_like.h:283-379).  CholeskyQR2 in FP64 on the GPU; R has a positive diagonal.
template <typename T>
LMatrix<T> tall_skinny_qr_factorize(DMatrix<T> A, int i1, int j1, int i2, int j2) {
  using namespace darray_b200::detail;
  const int m = i2 - i1, n = j2 - j1;
  assert(m > n);
  T* a = A.data() + i1 + (size_t)j1 * A.lld();
  Dev<double> dy((size_t)m * n), dr((size_t)n * n);
  upload(dy, a, m, n, A.lld());
  check(db200_cholqr2(ctx(), m, n, dy.p, m, dr.p, n), "tall_skinny_qr_factorize");
  download(a, m, n, A.lld(), dy);
  LMatrix<T> R(n, n);
  download(R.data(), n, n, R.ld(), dr);
  return R;
}

// Singular values of the (square) LMatrix, descending, as an m x 1 LMatrix (include/lapack_like.h:389-413).
template <typename T>
LMatrix<T> svd(int rank, LMatrix<T> LA, int i1, int j1, int i2, int j2) {
  (void)rank;
  (void)i1;
  (void)j1;
  (void)i2;
  (void)j2;
  using namespace darray_b200::detail;
  const int m = LA.dims()[0], n = LA.dims()[1];
  assert(m == n);
  Dev<double> da((size_t)m * n), ds(m);
  upload(da, LA.data(), m, n, LA.ld());
  check(db200_svd_values(ctx(), m, da.p, m, ds.p), "svd");
  LMatrix<T> S(m, 1);
  download(S.data(), m, 1, m, ds);
  return S;
}

}  // namespace DArray
