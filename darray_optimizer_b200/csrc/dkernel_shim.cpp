// Drop-in replacement for the reference's prebuilt include/dkernel.o: the same C++-linkage entry points with the
// same signatures (include/dkernel.h:6-8, include/dkernel.cu:28-38, include/dbarrier.cu:80), implemented over the
// C ABI.  Like the reference they take HOST pointers, copy to the device, compute and copy back, and stop the
// process with a message on a GPU error (include/dkernel.cu:20-26); unlike it they cover every block and honour
// beta and the leading dimensions.
#include <cstdio>
#include <cstdlib>

#include "internal.h"

#define DB200_CXX_API __attribute__((visibility("default")))

namespace {

db200_context* ctx_or_die() {
  db200_context* c = db200_default_context();
  if (!c) {
    std::fprintf(stderr, "darray_b200: no usable sm_100 device for the default context\n");
    std::exit(EXIT_FAILURE);
  }
  return c;
}

void check(db200_context* c, int st, const char* where) {
  if (st != DB200_OK) {
    std::fprintf(stderr, "darray_b200: %s failed: %s (status %d)\n", where, db200_last_error(c), st);
    std::exit(st < 0 ? -st : st);
  }
}

// RAII device buffer through the C ABI
struct DevBuf {
  db200_context* c;
  void* p = nullptr;
  DevBuf(db200_context* ctx, size_t bytes) : c(ctx) { check(c, db200_malloc(c, bytes, &p), "device allocation"); }
  ~DevBuf() { db200_free(c, p); }
  template <class T>
  T* as() { return static_cast<T*>(p); }
};

// copy an m x n column-major host block (leading dimension ld) into a packed device buffer: one copy, strided
// (cudaMemcpy2DAsync) when ld > m
template <class T>
void up(db200_context* c, T* dst, const T* src, int m, int n, int ld) {
  if (ld == m) {
    check(c, db200_copy_to_device(c, dst, src, sizeof(T) * (size_t)m * n), "copy to device");
    return;
  }
  if (cudaMemcpy2DAsync(dst, sizeof(T) * (size_t)m, src, sizeof(T) * (size_t)ld, sizeof(T) * (size_t)m, (size_t)n,
                        cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    check(c, DB200_ERR_CUDA, "copy to device");
}
template <class T>
void down(db200_context* c, T* dst, int ld, const T* src, int m, int n) {
  if (ld == m) {
    check(c, db200_copy_to_host(c, dst, src, sizeof(T) * (size_t)m * n), "copy to host");
    return;
  }
  if (cudaMemcpy2DAsync(dst, sizeof(T) * (size_t)ld, src, sizeof(T) * (size_t)m, sizeof(T) * (size_t)m, (size_t)n,
                        cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
    check(c, DB200_ERR_CUDA, "copy to host");
  check(c, db200_synchronize(c), "copy to host");
}

}  // namespace

// cuda_init (include/dkernel.cu:28-35): sets up the process-wide context (handles + stream).
DB200_CXX_API void cuda_init() { ctx_or_die(); }

// cuda_finalize (include/dkernel.cu:38-39): releases it.
DB200_CXX_API void cuda_finalize() { db200_release_default_context(); }

// rbf_kernel (include/dkernel.cu:132-190): K(m x n, ldk) = diag(Yi) exp(-gamma D2(Xi, Xj)) diag(Yj), with Xi
// (m x d) and Xj (n x d) column major (ldxi >= m, ldxj >= n), all host pointers.
DB200_CXX_API void rbf_kernel(int rank, int m, int n, int d, float* Xi, int ldxi, float* Xj, int ldxj, float* Yi,
                              float* Yj, float* K, int ldk, float gamma) {
  (void)rank;
  if (m <= 0 || n <= 0) return;
  db200_context* c = ctx_or_die();
  DevBuf xi(c, sizeof(float) * (size_t)m * d), xj(c, sizeof(float) * (size_t)n * d);
  DevBuf yi(c, sizeof(float) * m), yj(c, sizeof(float) * n), k(c, sizeof(float) * (size_t)m * n);
  up(c, xi.as<float>(), Xi, m, d, ldxi);
  up(c, xj.as<float>(), Xj, n, d, ldxj);
  check(c, db200_copy_to_device(c, yi.p, Yi, sizeof(float) * m), "copy to device");
  check(c, db200_copy_to_device(c, yj.p, Yj, sizeof(float) * n), "copy to device");
  check(c, db200_rbf_block(c, m, n, d, xi.as<float>(), m, xj.as<float>(), n, DB200_FEATURE_MAJOR, yi.as<float>(),
                           yj.as<float>(), k.as<float>(), m, gamma),
        "rbf_kernel");
  down(c, K, ldk, k.as<float>(), m, n);
}

// tc_gemm (include/dkernel.cu:194-231): C(m x k) = alpha A(m x n) B(n x k) + beta C, host pointers.
DB200_CXX_API void tc_gemm(int rank, int m, int k, int n, float* A, int lda, float* BB, int ldb, float* C, int ldc,
                           float alpha, float beta) {
  (void)rank;
  if (m <= 0 || k <= 0) return;
  db200_context* c = ctx_or_die();
  DevBuf a(c, sizeof(float) * (size_t)m * n), b(c, sizeof(float) * (size_t)n * k), cc(c, sizeof(float) * (size_t)m * k);
  up(c, a.as<float>(), A, m, n, lda);
  up(c, b.as<float>(), BB, n, k, ldb);
  if (beta != 0.0f) up(c, cc.as<float>(), C, m, k, ldc);
  check(c, db200_sgemm(c, 'N', 'N', m, k, n, alpha, a.as<float>(), m, b.as<float>(), n, beta, cc.as<float>(), m),
        "tc_gemm");
  down(c, C, ldc, cc.as<float>(), m, k);
}

// tc_sgemm (include/dkernel.cu:234-275): C(m x k) = alpha op(A) B + beta C with op(A) = A (m x n) or A^T (A is
// n x m), host pointers.
DB200_CXX_API void tc_sgemm(int rank, char transA, char transB, int m, int k, int n, float* A, int lda, float* BB,
                            int ldb, float* C, int ldc, float alpha, float beta) {
  (void)rank;
  if (m <= 0 || k <= 0) return;
  db200_context* c = ctx_or_die();
  const bool ta = (transA == 'T' || transA == 't');
  const int ar = ta ? n : m, ac = ta ? m : n;
  DevBuf a(c, sizeof(float) * (size_t)ar * ac), b(c, sizeof(float) * (size_t)n * k), cc(c, sizeof(float) * (size_t)m * k);
  up(c, a.as<float>(), A, ar, ac, lda);
  up(c, b.as<float>(), BB, n, k, ldb);
  if (beta != 0.0f) up(c, cc.as<float>(), C, m, k, ldc);
  check(c, db200_sgemm(c, transA, transB, m, k, n, alpha, a.as<float>(), ar, b.as<float>(), n, beta, cc.as<float>(),
                       m),
        "tc_sgemm");
  down(c, C, ldc, cc.as<float>(), m, k);
}

// logbarrier (include/dbarrier.cu:80-87): the reference body only allocates device buffers and returns; the
// barrier solve itself is db200_svm_barrier.  Kept so that callers linking the symbol still link.
DB200_CXX_API void logbarrier(double* K, int ldk, int m, int n) {
  (void)K;
  (void)ldk;
  (void)m;
  (void)n;
}
