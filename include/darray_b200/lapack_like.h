// One-rank mirror of include/lapack_like.h on the GPU: cholesky_factorize, cholesky_factorize_recursive,
// tall_skinny_qr_factorize and svd (FP64 arithmetic on float or double DMatrix data), and the LU factorisations
// lu_factorize_partial_pivot, lu_factorize_partial_pivot_replicate_panel, lu_factorize_no_pivot and
// lu_factorize_unblocked (FP32, db200_lu_factorize).
#pragma once
#include <algorithm>
#include <cassert>
#include <type_traits>
#include <vector>

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

namespace lu_detail {
// LU of the m x n block at (i, j) on the GPU; the row interchanges also reach the `left` columns [j - left, j).
// Sets A.ipiv()[i + k] to the 1-based global pivot rows when record_ipiv.
inline std::vector<int> lu_block(DMatrix<float>& A, int i, int j, int m, int n, int left, int pivot, int swap_left,
                                 bool record_ipiv) {
  using namespace darray_b200::detail;
  const int mn = std::min(m, n), cols = left + n;
  std::vector<int> ipiv(mn, 0);
  if (m <= 0 || n <= 0) return ipiv;
  float* a = A.data() + i + (size_t)(j - left) * A.lld();
  Dev<float> d((size_t)m * cols);
  Dev<int> dp(mn);
  upload(d, a, m, cols, A.lld());
  check(db200_lu_factorize(ctx(), m, n, left, d.p + (size_t)left * m, m, dp.p, pivot, swap_left),
        "lu_factorize");
  download(a, m, cols, A.lld(), d);
  check(db200_copy_to_host(ctx(), ipiv.data(), dp.p, sizeof(int) * mn), "copy to host");
  if (record_ipiv)
    for (int k = 0; k < mn; ++k) A.ipiv()[i + k] = ipiv[k] + i;
  return ipiv;
}
}  // namespace lu_detail

// LU with partial pivoting of A[i:i+m, j:j+n] in place (include/lapack_like.h:179-219): L unit lower below the
// diagonal, U on and above it; A.ipiv() gets the 1-based global pivot rows, and the rows are interchanged in the
// columns left of the block too, as the reference does.  bs (the reference's outer block) does not change the
// result beyond rounding: the GPU blocks by 32.  FP32 only, as the reference (its sgetrf/strsm/sgemm calls).
template <typename T>
void lu_factorize_partial_pivot(DMatrix<T>& A, int i, int j, int m, int n, int bs = 256) {
  static_assert(std::is_same<T, float>::value, "lu_factorize_partial_pivot: float, as the reference's BLAS calls");
  (void)bs;
  assert(i + m <= A.dims()[0] && j + n <= A.dims()[1]);
  lu_detail::lu_block(A, i, j, m, n, j, 1, 1, true);
}

// The replicate-panel variant (include/lapack_like.h:134-177): each panel's interchanges reach only the columns
// right of it, so the L of earlier panels is left in the order it was computed in.  (The reference's template
// does not compile when instantiated, lapack_like.h:152; this follows what its code describes.)
template <typename T>
void lu_factorize_partial_pivot_replicate_panel(DMatrix<T>& A, int i, int j, int m, int n, int bs = 256) {
  static_assert(std::is_same<T, float>::value, "lu_factorize_partial_pivot_replicate_panel: float");
  (void)bs;
  assert(i + m <= A.dims()[0] && j + n <= A.dims()[1]);
  lu_detail::lu_block(A, i, j, m, n, 0, 1, 0, true);
}

// LU without interchanges (include/lapack_like.h:93-131; A.ipiv() untouched).  The reference factors each diagonal
// block with sgetrf, which may pivot inside the block while the rest of the matrix is not permuted; here no row
// is ever exchanged, which is what the two agree on for the diagonally dominant matrices it is meant for.
template <typename T>
void lu_factorize_no_pivot(DMatrix<T>& A, int i, int j, int m, int n, int bs = 256) {
  static_assert(std::is_same<T, float>::value, "lu_factorize_no_pivot: float");
  (void)bs;
  assert(i + m <= A.dims()[0] && j + n <= A.dims()[1]);
  lu_detail::lu_block(A, i, j, m, n, 0, 0, 0, false);
}

// Unblocked LU of A[i1:i2, j1:j2] (include/lapack_like.h:220-279): interchanges only inside those columns, the
// pivots returned 1-based relative to i1.
template <typename T>
std::vector<int> lu_factorize_unblocked(DMatrix<T> A, int i1, int j1, int i2, int j2) {
  static_assert(std::is_same<T, float>::value, "lu_factorize_unblocked: float");
  return lu_detail::lu_block(A, i1, j1, i2 - i1, j2 - j1, 0, 1, 1, false);
}

}  // namespace DArray
