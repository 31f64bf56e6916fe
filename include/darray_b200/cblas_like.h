// One-rank mirror of include/cblas_like.h's LMatrix wrappers (multiply_matrix, symmetric_update) on the GPU.
// The Fortran BLAS prototypes of the reference are not needed: every product runs through libdarray_b200.
#pragma once
#include "darray.h"
#include "detail.h"

namespace DArray {

// C = alpha op(A) op(B) + beta C (include/cblas_like.h:40-60), FP64 accumulation for float and double.
template <typename T>
void multiply_matrix(const char* ta, const char* tb, T alpha, T beta, LMatrix<T>& A, LMatrix<T>& B, LMatrix<T>& C) {
  using namespace darray_b200::detail;
  const bool tA = (*ta == 'T' || *ta == 't'), tB = (*tb == 'T' || *tb == 't');
  const int m = C.dims()[0], n = C.dims()[1], k = tA ? A.dims()[0] : A.dims()[1];
  assert((tA ? A.dims()[1] : A.dims()[0]) == m && (tB ? B.dims()[0] : B.dims()[1]) == n);
  const int ar = A.dims()[0], ac = A.dims()[1], br = B.dims()[0], bc = B.dims()[1];
  Dev<double> da((size_t)ar * ac), db((size_t)br * bc), dc((size_t)m * n);
  upload(da, A.data(), ar, ac, A.ld());
  upload(db, B.data(), br, bc, B.ld());
  if (beta != T(0)) upload(dc, C.data(), m, n, C.ld());
  check(db200_gemm(ctx(), *ta, *tb, m, n, k, (double)alpha, da.p, ar, db.p, br, (double)beta, dc.p, m), "multiply_matrix");
  download(C.data(), m, n, C.ld(), dc);
}

// A22 <- A22 - A12^T A12 on the upper triangle (include/cblas_like.h:62-69: ssyrk with -1 and 1; like the
// reference, the alpha and beta arguments are not used).
template <typename T>
void symmetric_update(const char* uplo, const char* trans, float alpha, LMatrix<T>& A12, float beta, LMatrix<T>& A22) {
  (void)uplo;
  (void)trans;
  (void)alpha;
  (void)beta;
  using namespace darray_b200::detail;
  const int k = A12.dims()[0], n = A22.dims()[0];
  Dev<double> da((size_t)k * n), dc((size_t)n * n);
  upload(da, A12.data(), k, n, A12.ld());
  upload(dc, A22.data(), n, n, A22.ld());
  check(db200_gemm(ctx(), 'T', 'N', n, n, k, -1.0, da.p, k, da.p, k, 1.0, dc.p, n), "symmetric_update");
  download(A22.data(), n, n, A22.ld(), dc, true);
}

}  // namespace DArray
