// One-rank mirror of include/dkernel.h (rushah05/DArray_Optimizer): the GPU entry points with the reference's
// C++ signatures (exported by libdarray_b200.so in place of include/dkernel.o) and DArray::LRA / DArray::Knorm
// over the fused B200 kernels.
#pragma once
#include "blas_like.h"
#include "darray.h"
#include "detail.h"

#define NN 50000  // out-of-core block of the reference (include/dkernel.h:4); kept for source compatibility

void rbf_kernel(int rank, int m, int n, int d, float* Xi, int ldxi, float* Xj, int ldxj, float* Yi, float* Yj, float* K,
                int ldk, float gamma);
void tc_gemm(int rank, int m, int k, int n, float* A, int lda, float* BB, int ldb, float* C, int ldc, float alpha = 1,
             float beta = 0);
void tc_sgemm(int rank, char transA, char transB, int m, int k, int n, float* A, int lda, float* BB, int ldb, float* C,
              int ldc, float alpha = 1, float beta = 0);
void cuda_init();
void cuda_finalize();
void logbarrier(double* K, int ldk, int m, int n);

namespace DArray {

// A(n x k) = diag(Y) K(X, X) diag(Y) O over the whole kernel (include/dkernel.h:13-46; the reference stops after
// its first block).  X is d x n, Y 1 x n, O and A n x k.
template <typename T>
void LRA(Grid g, int n, int d, int k, DMatrix<T> X, DMatrix<T>& Y, DMatrix<T>& O, DMatrix<T>& A, float gamma) {
  static_assert(sizeof(T) == sizeof(float), "LRA is provided for DMatrix<float>, as in the reference");
  (void)g;
  using namespace darray_b200::detail;
  check(db200_lra_host(ctx(), n, d, k, X.data(), X.lld(), Y.data(), O.data(), O.lld(), A.data(), A.lld(), gamma), "LRA");
}

// Prints ||K||_F, ||K - Z Z^T||_F and their ratio (include/dkernel.h:50-76, corrected to measure K - Z Z^T over
// every block); returns the ratio.
template <typename T>
double Knorm(Grid g, int n, int d, int k, DMatrix<T>& X, DMatrix<T>& Y, DMatrix<T>& Z, float gamma) {
  using namespace darray_b200::detail;
  Dev<float> dx((size_t)n * d), dy(n);
  Dev<double> dz((size_t)n * k);
  upload(dx, X.data(), d, n, X.lld());
  upload(dy, Y.data(), 1, n, 1);
  upload(dz, Z.data(), n, k, Z.lld());
  double out[3];
  check(db200_knorm(ctx(), n, d, k, dx.p, d, dy.p, dz.p, n, gamma, out), "Knorm");
  if (g.rank() == 0) std::printf("fnorm(K)=%f fnorm(K-U*U)=%f Residual fnorm=%f\n", out[0], out[1], out[2]);
  return out[2];
}

}  // namespace DArray
