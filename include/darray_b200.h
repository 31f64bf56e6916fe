/*
 * darray_b200.h -- C ABI of libdarray_b200.so, the B200 (sm_100a) implementation of DArray's
 * kernel-SVM hot path (rushah05/DArray_Optimizer).
 *
 * Conventions
 *   - Every function returns an int status (DB200_OK == 0, negative on error); the message of the last
 *     error is available from db200_last_error().
 *   - Matrices are column-major with an explicit leading dimension, as in the reference's LMatrix/DMatrix.
 *   - "Device" entry points take device pointers and are stream-ordered on the context's stream; they do
 *     not synchronize.  db200_synchronize() waits and also reports errors raised inside kernels (a bounded
 *     device-side wait that gave up reports DB200_ERR_TIMEOUT).
 *   - No torch or C++ types cross this boundary.
 */
#ifndef DARRAY_B200_H
#define DARRAY_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DB200_API __attribute__((visibility("default")))
#else
#define DB200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define DB200_OK 0
#define DB200_ERR_INVALID (-1)     /* bad argument (size, pointer, leading dimension) */
#define DB200_ERR_CUDA (-2)        /* CUDA runtime/driver error */
#define DB200_ERR_NOT_SPD (-3)     /* Cholesky met a non-positive pivot */
#define DB200_ERR_MAXITER (-4)     /* an iteration cap was reached */
#define DB200_ERR_INFEASIBLE (-5)  /* barrier iterate left the box 0 < a < C */
#define DB200_ERR_TIMEOUT (-6)     /* a bounded device-side wait gave up */
#define DB200_ERR_NOMEM (-7)       /* device allocation failed */
#define DB200_ERR_UNSUPPORTED (-8) /* shape outside what the kernels implement */
#define DB200_ERR_TOO_LARGE (-9)   /* request exceeds the fixed scratch of db200_rbf_sketch_noalloc */

/* Layout of a point matrix X holding n points of d features. */
#define DB200_POINT_MAJOR 0   /* x(i,k) = X[k + i*ldx]  (the reference's DMatrix X, d x n column major) */
#define DB200_FEATURE_MAJOR 1 /* x(i,k) = X[i + k*ldx]  (rbf_kernel's Xi/Xj, m x d column major) */

typedef struct db200_context db200_context;

/* Pass as `stream` to db200_create() to have the context create (and later destroy) its own stream. */
#define DB200_OWN_STREAM ((void*)(intptr_t)-1)

/* Create a context on `device`.  `stream` is the cudaStream_t all work is queued on (NULL: the CUDA default
 * stream; DB200_OWN_STREAM: a new non-blocking stream owned by the context).
 * Replaces cuda_init() (include/dkernel.cu:28), whose handles were process globals. */
DB200_API int db200_create(db200_context** ctx, int device, void* stream);

/* Release the context and its device workspace.  Replaces cuda_finalize() (include/dkernel.cu:38). */
DB200_API int db200_destroy(db200_context* ctx);

/* Message of the last error on this context ("" if none). */
DB200_API const char* db200_last_error(const db200_context* ctx);

/* Wait for all work queued on the context's stream; returns the first device-side error if any. */
DB200_API int db200_synchronize(db200_context* ctx);

/* The context's stream as a cudaStream_t. */
DB200_API void* db200_stream(const db200_context* ctx);

/* Number of kernels this library has launched on this context since creation (launch accounting). */
DB200_API int64_t db200_launch_count(const db200_context* ctx);

/* Enable (1) or disable (0) CUDA-event timing of every tcgen05 tile-kernel launch on the context's stream;
 * db200_profile_read() returns the summed kernel time (ms) and the number of timed launches since the last
 * read, then clears them.  Both synchronize the stream. */
DB200_API int db200_profile(db200_context* ctx, int enable);
DB200_API int db200_profile_read(db200_context* ctx, double* total_ms, int64_t* count);

/*
 * Fused RBF kernel x sketch (device pointers):
 *     Y(m x l) = diag(yi) * K(Xi, Xj) * diag(yj) * Omega,   K(a,b) = exp(-gamma * ||x_a - x_b||^2)
 * The kernel block K is never stored: squared distances come from split-bf16 tensor-core products
 * (||x||^2 + ||y||^2 - 2 x.y), exp is applied in the epilogue and the bf16 tile feeds the sketch product,
 * accumulated in fp32.  Replaces rbf_kernel (include/dkernel.cu:132) followed by tc_gemm
 * (include/dkernel.cu:194) inside DArray::LRA (include/dkernel.h:13-46), for the whole n x n matrix.
 *   Xi, Xj : points in `x_layout` (DB200_POINT_MAJOR or DB200_FEATURE_MAJOR) with leading dims ldxi/ldxj
 *   yi, yj : labels of length m and n (NULL means all ones)
 *   Omega  : n x l column major (ldo >= n);  Y : m x l column major (ldy >= m)
 * Supports d <= 128.
 */
DB200_API int db200_rbf_sketch(db200_context* ctx, int m, int n, int d, int l, const float* Xi, int ldxi, const float* Xj,
                     int ldxj, int x_layout, const float* yi, const float* yj, const float* Omega, int ldo, float* Y,
                     int ldy, float gamma);

/*
 * Materialised RBF block (device pointers):  K(m x n) = diag(yi) * exp(-gamma * D2(Xi, Xj)) * diag(yj),
 * column major with leading dimension ldk.  Same arithmetic as db200_rbf_sketch's epilogue, in fp32.
 * Replaces rbf_kernel (include/dkernel.cu:132-190, kernels vecnorm :102 and rbf :116) on device memory.
 */
DB200_API int db200_rbf_block(db200_context* ctx, int m, int n, int d, const float* Xi, int ldxi, const float* Xj, int ldxj,
                    int x_layout, const float* yi, const float* yj, float* K, int ldk, float gamma);

/*
 * Host-pointer sketch with the calling convention of DArray::LRA (include/dkernel.h:13) on a 1 x 1 grid:
 *     A(n x k) = diag(Y) K(X, X) diag(Y) O
 * X is the d x n feature matrix (column major, ldx >= d: the reference's DMatrix X of tests/testsvm.cpp:76),
 * Y the n labels, O the n x k test matrix (ldo >= n), A the n x k result (lda >= n).  Copies in, runs the fused
 * kernel over every block (the reference stops after the first, include/dkernel.h:43) and copies out;
 * synchronous.  Stands in for the rbf_kernel + tc_gemm host round trips of include/dkernel.cu:132-231.
 */
DB200_API int db200_lra_host(db200_context* ctx, int n, int d, int k, const float* X, int ldx, const float* Y,
                             const float* O, int ldo, float* A, int lda, float gamma);

/* ------------------------------------------------------------------------------------------------------
 * Dense FP64 linear algebra on a 1 x 1 DMatrix (device pointers, column major).
 * ------------------------------------------------------------------------------------------------------ */

/* In-place upper Cholesky A = R^T R of the n x n matrix A (only the upper triangle is read; the strictly lower
 * part is zeroed), blocked right-looking with block size nb (<= 64; 0 = 64).  A non-positive pivot returns
 * DB200_ERR_NOT_SPD (db200_last_error names the failing block).  Replaces cholesky_factorize(A, 'U', n, 0, bs)
 * and cholesky_factorize_recursive (include/lapack_like.h:10-90), in FP64.  Synchronous. */
DB200_API int db200_potrf(db200_context* ctx, int n, double* A, int lda, int nb);

/* Orthonormalise the tall-skinny Y (n x l, n >= l) in place by CholeskyQR2 (FP64 Gram Y^T Y, Cholesky,
 * Y <- Y R^-1, twice; falls back to shifted CholeskyQR3 when the first Gram is numerically singular) and
 * return R (l x l upper, Y_in = Q R, positive diagonal).  Replaces tall_skinny_qr_factorize
 * (include/lapack_like.h:283-379), which returns R and overwrites A with Q.  Synchronous. */
DB200_API int db200_cholqr2(db200_context* ctx, int n, int l, double* Y, int ldy, double* R, int ldr);

/* C(m x n) = alpha * A^T B + beta * C with A k x m and B k x n, FP64.  Replaces matrix_multiply("T","N")
 * (include/blas_like.h:63-93) and multiply_matrix (include/cblas_like.h:40-60). */
DB200_API int db200_gemm_tn(db200_context* ctx, int k, int m, int n, double alpha, const double* A, int lda,
                            const double* B, int ldb, double beta, double* C, int ldc);

/* B(m x n) <- U^-T B with U the upper triangle of the m x m matrix R.  Replaces triangular_solve("L","U","T","N")
 * (include/blas_like.h:96-127). */
DB200_API int db200_trsm_lutn(db200_context* ctx, int m, int n, const double* R, int ldr, double* B, int ldb);

/* ------------------------------------------------------------------------------------------------------
 * Kernel SVM: low-rank factor and barrier solve.
 * ------------------------------------------------------------------------------------------------------ */

/* Barrier-method constants, defaults from tests/testsvm.cpp:228-321 (t0 = 1, mu = 20, alpha = 0.1,
 * beta = 0.5, Newton stop lambda^2/2 < 1e-6) with the barrier stop 2n/t < gap_tol * |f(a)|, gap_tol = 1e-6. */
typedef struct db200_barrier_params {
  double t0, mu, alpha, beta, gap_tol, newton_tol;
  int max_outer, max_newton;
} db200_barrier_params;

/* What a solve did and where it ended. */
typedef struct db200_svm_report {
  double f;                /* dual objective f(a) = 0.5 a^T Z Z^T a - 1^T a at the returned a */
  double gap_barrier;      /* 2n/t / |f|: the barrier method's duality-gap bound */
  double gap_primal_dual;  /* (P(Z^T a) + f(a)) / |f|, P(w) = 0.5|w|^2 + C sum max(0, 1 - z_i.w) */
  double t;                /* final barrier parameter */
  double nu;               /* shift of the Nystrom core Cholesky */
  int outer, newton;       /* barrier and Newton iterations */
  int status;              /* DB200_OK, DB200_ERR_MAXITER (caps reached) */
  double ms_sketch, ms_orth, ms_core, ms_barrier, ms_total;
} db200_svm_report;

DB200_API void db200_barrier_defaults(db200_barrier_params* p);

/* Minimise f(a) = 0.5 a^T Z Z^T a - 1^T a over 0 < a < C by the log-barrier method with Newton steps solved
 * through Sherman-Morrison-Woodbury on the r x r capacity matrix I + Z^T D^-1 Z (FP64 Cholesky), line search
 * kept inside the box.  Z: n x r FP64 (labels folded in, z_i = y_i phi(x_i)), y: n labels (float, +-1) for the
 * class-balanced start of tests/testsvm.cpp:192-212, a: n FP64 output.  Replaces the loop of
 * tests/testsvm.cpp:228-321 over include/dbarrier.h:14-139 (f, gg, Grad_f, Grad_Phi, Grad, Hess_Phi,
 * pre_conjgrad).  Synchronous; rep may be NULL. */
DB200_API int db200_svm_barrier(db200_context* ctx, int n, int r, const double* Z, int ldz, const float* y, double C,
                                const db200_barrier_params* p, double* a, db200_svm_report* rep);

/* Low-rank factor Z (n x l FP64, Z Z^T ~ diag(y) K diag(y)) by the randomised range finder of
 * tests/testsvm.cpp:86-170, corrected: Y = K Omega; Q = orth(Y); q times {Y = K Q; Q = orth(Y)};
 * C = Q^T K Q; R^T R = C + nu I; Z = Q R^T.  K products use the fused kernel (db200_rbf_sketch), orth is
 * db200_cholqr2.  X point-major (ldx >= d), y and Omega (n x l, ldo >= n) device.  Synchronous. */
DB200_API int db200_lowrank(db200_context* ctx, int n, int d, int l, int q, const float* X, int ldx, const float* y,
                            const float* Omega, int ldo, float gamma, double* Z, int ldz, db200_svm_report* rep);

/* The whole path: db200_lowrank followed by db200_svm_barrier (tests/testsvm.cpp:34-329 at one rank).
 * Outputs a (n, FP64) and Z (n x l FP64).  Synchronous; rep may be NULL. */
DB200_API int db200_svm_solve(db200_context* ctx, int n, int d, int l, int q, const float* X, int ldx,
                              const float* y, const float* Omega, int ldo, float gamma, double C,
                              const db200_barrier_params* p, double* a, double* Z, int ldz, db200_svm_report* rep);

/*
 * Allocation-free fused RBF x sketch.  No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc -- plugin hosts that own every device allocation and only lend a stream, processes under a hard
 * memory budget, or latency-critical phases that must not enter the allocator.
 *
 * Same arguments, arithmetic and result as db200_rbf_sketch, but no context: work is queued on `stream`
 * (a cudaStream_t; NULL = the default stream) and the call waits for it before returning.  Its scratch
 * (packed operands and a status word) is one static device array of DB200_NOALLOC_SCRATCH_BYTES that every GPU
 * loading this library holds until the process exits; the function calls no cudaMalloc, cudaFree or other
 * allocating routine.  Requests whose scratch would exceed the array return DB200_ERR_TOO_LARGE (with a message
 * on stderr naming the bytes needed).  The scratch need is about
 *     (m + n) * (4 * roundup(d, 32) + 4) + 2 * n * roundup(l, 16)   bytes   (the n term once when Xi == Xj).
 * The first call on each device resolves the array's device address (cudaGetSymbolAddress, with that device
 * current); make that first call before any stream capture.  All calls share the one array and it keeps the
 * previous call's contents (every byte a call reads is written by that call first); calls that overlap on the
 * GPU -- from two host threads, or on two streams -- race on it and must be serialised by the caller.
 */
#define DB200_NOALLOC_SCRATCH_BYTES (32u << 20)
DB200_API int db200_rbf_sketch_noalloc(void* stream, int m, int n, int d, int l, const float* Xi, int ldxi,
                                       const float* Xj, int ldxj, int x_layout, const float* yi, const float* yj,
                                       const float* Omega, int ldo, float* Y, int ldy, float gamma);

#ifdef __cplusplus
}
#endif

#endif /* DARRAY_B200_H */
