// C entry points over the reference's own GPU kernel-block code (include/dkernel.cu, compiled unmodified
// beside this file by oracle/build_ref.sh into oracle/_ref/libdkernel_ref.so).  Test infrastructure only:
// the product never links it.  The reference exports C++ symbols, so ctypes needs these unmangled wrappers.
//
// The reference's behaviour is kept as it is, including what a caller has to know:
//   * rbf_kernel (include/dkernel.cu:132-190) takes column-major host buffers and ignores ldxi/ldxj: Xi is
//     read with leading dimension m and Xj with n (include/dkernel.cu:153,161);
//   * tc_gemm (include/dkernel.cu:194-231) passes beta = 0 to every 8192-column block, so for n > 8192
//     only the last block's product survives; results are only meaningful for n <= 8192;
//   * the first call needs ref_cuda_init() (include/dkernel.cu:28-34), which creates the global cuBLAS
//     handle and stream.

void cuda_init();
void rbf_kernel(int rank, int m, int n, int d, float* Xi, int ldxi, float* Xj, int ldxj, float* Yi, float* Yj,
                float* K, int ldk, float gamma);
void tc_gemm(int rank, int m, int k, int n, float* A, int lda, float* BB, int ldb, float* C, int ldc, float alpha,
             float beta);

extern "C" {

void ref_cuda_init() { cuda_init(); }

// K (m x n, column-major, leading dimension ldk) = diag(Yi) exp(-gamma ||xi - xj||^2) diag(Yj).
void ref_rbf_kernel(int m, int n, int d, float* Xi, float* Xj, float* Yi, float* Yj, float* K, int ldk,
                    float gamma) {
  rbf_kernel(0, m, n, d, Xi, m, Xj, n, Yi, Yj, K, ldk, gamma);
}

// C (m x k) = alpha A (m x n) B (n x k), all column-major host buffers.
void ref_tc_gemm(int m, int k, int n, float* A, int lda, float* Bm, int ldb, float* C, int ldc, float alpha) {
  tc_gemm(0, m, k, n, A, lda, Bm, ldb, C, ldc, alpha, 0.0f);
}

}  // extern "C"
