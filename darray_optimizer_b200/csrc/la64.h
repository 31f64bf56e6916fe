// FP64 dense linear-algebra building blocks (la64.cu).  All stream-ordered on ctx->stream, column major.
#pragma once
#include "internal.h"

namespace db200 {

// C[p x q] = alpha * A^T diag(w) B + beta * C over n rows (w may be null); FP64 accumulation.  With upper_only
// only the upper triangle of C (p == q) is formed.  Restates matrix_multiply("T","N") of include/blas_like.h:63.
template <typename TA, typename TBt>
int gram(db200_context* ctx, int n, int p, int q, const TA* A, long long lda, const TBt* B, long long ldb,
         const double* w, double alpha, double beta, double* C, int ldc, bool upper_only);

// C[n x q] = A[n x p] * op(B) + beta * C,  op(B) = B (p x q, ldb) or B^T (B stored q x p) when transB.
template <typename TA, typename TC>
int gemm_tall(db200_context* ctx, int n, int p, int q, const TA* A, long long lda, const double* B, int ldb,
              bool transB, double beta, TC* C, long long ldc, double alpha = 1.0);

// In-place upper Cholesky (A = R^T R) with block size nb <= 64; the strictly lower part is zeroed.  A
// non-positive pivot sets *d_status = DB200_ERR_NOT_SPD and *d_bad = first row of the failing block.
// Restates cholesky_factorize(A, 'U', n, 0, bs) of include/lapack_like.h:10-56.
int potrf_upper(db200_context* ctx, double* A, int lda, int l, int* d_status, int* d_bad, int nb = 64);

// The same factor in one launch on a thread-block cluster for 1 <= l <= 544 (potrf_cluster.cu); returns
// DB200_ERR_UNSUPPORTED, launching nothing, where no cluster configuration holds the matrix.  potrf_cluster_init
// probes the device's largest cluster once (outside any stream capture); potrf_cluster_size gives the cluster size
// used for l (0: none).
void potrf_cluster_init(db200_context* ctx);
int potrf_cluster_size(const db200_context* ctx, int l);
int potrf_cluster(db200_context* ctx, double* A, int lda, int l, int* d_status, int* d_bad);

// X = R^-1 for upper triangular R.
int trinv_upper(db200_context* ctx, const double* R, int ldr, int l, double* X, int ldx);

// In-place triangular solve with upper R and its stored transpose L: transposed -> R^T x = b, else R x = b.
int trsv_upper(db200_context* ctx, const double* R, const double* L, int ld, int l, double* x, bool transposed);

int transpose64(db200_context* ctx, const double* A, int lda, int m, int n, double* B, int ldb);
int symmetrize(db200_context* ctx, double* C, int ldc, int l, double shift);
int mirror_upper(db200_context* ctx, double* C, int ldc, int l);
template <typename TS, typename TD>
int convert(db200_context* ctx, const TS* src, long long lds, TD* dst, long long ldd, int m, int n);
int trace(db200_context* ctx, const double* C, int ldc, int l, double* d_out);
// C (float) = alpha * T (double) + beta * C
int axpby_f32(db200_context* ctx, float* C, long long ldc, const double* T, long long ldt, int m, int n,
              double alpha, double beta);
// *d_out += sum of squares of an m x n float block
int sumsq_f32(db200_context* ctx, const float* A, long long lda, int m, int n, double* d_out);
// K = yi yj exp(-gamma max(si + sj - 2 G, 0)) in place over an m x n FP64 Gram block
int rbf_from_gram_f64(db200_context* ctx, double* K, long long ldk, int m, int n, const double* si, const double* sj,
                      const float* yi, const float* yj, double gamma);
// FP64 squared norms of the n points of a point-major float matrix
int rownorm_f64(db200_context* ctx, const float* X, long long ldx, int n, int d, double* s);
// Fused FP64 RBF x sketch (rbf64.cu): Y = diag(yi) K(Xi, Xj) diag(yj) Omega, FP64 throughout, K never stored.
int rbf_sketch_f64_fused(db200_context* ctx, int m, int n, int d, int l, const float* Xi, int ldxi, const float* Xj,
                         int ldxj, const float* yi, const float* yj, const double* Omega, int ldo, double* Y, int ldy,
                         double gamma);
// sort descending, n <= 8192
int sort_desc(db200_context* ctx, double* v, int n);

// Singular values of the n x n matrix A (destroyed) by one-sided Jacobi, unsorted; *d_status = 1 if the sweep
// cap was reached.  Restates svd (include/lapack_like.h:389-413), which returns only S.
int jacobi_svd_values(db200_context* ctx, double* A, int lda, int n, double* S, int* d_status);

}  // namespace db200
