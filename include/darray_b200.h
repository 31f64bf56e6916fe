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
#define DB200_ERR_SINGULAR (-10)   /* LU met a zero pivot */
#define DB200_ERR_COLLECTIVE (-11) /* the collective set by db200_set_collective reported a failure */

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

/* Failure-path self-test of the bounded device waits: queues a kernel that waits on a flag nothing sets and
 * gives up after limit_ms (1..5000).  The next db200_synchronize returns DB200_ERR_TIMEOUT and clears it; the
 * context remains usable.  Stream-ordered. */
DB200_API int db200_selftest_wait_timeout(db200_context* ctx, int limit_ms);
/* The same for the grid-wide barrier of the cooperative LU panel (db200_lu_factorize): four co-resident CTAs of
 * which one never arrives; the other three give up after limit_ms (1..5000) and the next db200_synchronize
 * returns DB200_ERR_TIMEOUT and clears it. */
DB200_API int db200_selftest_grid_barrier_timeout(db200_context* ctx, int limit_ms);

/* Enable (1) or disable (0) CUDA-event timing of every tcgen05 tile-kernel launch on the context's stream;
 * db200_profile_read() returns the summed kernel time (ms) and the number of timed launches since the last
 * read, then clears them.  Both synchronize the stream. */
DB200_API int db200_profile(db200_context* ctx, int enable);
DB200_API int db200_profile_read(db200_context* ctx, double* total_ms, int64_t* count);

/* Measured FP64 throughput of this GPU in TFLOP/s: back-to-back mma.sync.m16n8k8.f64 (the FP64 tensor-core tiles
 * of the FP64 kernels) and back-to-back FP64 FMAs, operands in registers, 32 warps per SM, timed with CUDA events
 * (~60 ms).  The denominator of the FP64 kernels' roofline fractions.  Synchronous. */
DB200_API int db200_probe_fp64_peak(db200_context* ctx, double* dmma_tflops, double* dfma_tflops);

/*
 * Fused RBF kernel x sketch (device pointers):
 *     Y(m x l) = diag(yi) * K(Xi, Xj) * diag(yj) * Omega,   K(a,b) = exp(-gamma * ||x_a - x_b||^2)
 * The kernel block K is never stored: squared distances come from split-fp16 tensor-core products on points
 * scaled by powers of two (||x||^2 + ||y||^2 - 2 x.y, 22 significant bits per coordinate), exp is applied in the
 * epilogue and the fp16 tile feeds the sketch product, accumulated in fp32.  Replaces rbf_kernel
 * (include/dkernel.cu:132) followed by tc_gemm (include/dkernel.cu:194) inside DArray::LRA
 * (include/dkernel.h:13-46), for the whole n x n matrix.
 *   Xi, Xj : points in `x_layout` (DB200_POINT_MAJOR or DB200_FEATURE_MAJOR) with leading dims ldxi/ldxj
 *   yi, yj : labels of length m and n (NULL means all ones)
 *   Omega  : n x l column major (ldo >= n);  Y : m x l column major (ldy >= m)
 * Supports d <= 128.  The sketch product is the single fp16 product (DB200_SKETCH_SINGLE below).
 */
DB200_API int db200_rbf_sketch(db200_context* ctx, int m, int n, int d, int l, const float* Xi, int ldxi, const float* Xj,
                     int ldxj, int x_layout, const float* yi, const float* yj, const float* Omega, int ldo, float* Y,
                     int ldy, float gamma);

/* Sketch products of db200_rbf_sketch_ex.
 * DB200_SKETCH_SINGLE: P . Omega~ with both in fp16 (11 significant bits each), fp32 accumulation.  Relative
 *   error of Y ~3e-4.
 * DB200_SKETCH_P_SPLIT: adds P_lo . Omega~, P_lo = fp16(P - fp16(P)), so the kernel values carry ~22 bits.
 * DB200_SKETCH_COMPENSATED: adds P_hi . Omega~_lo as well (Omega~ also hi + lo): ~22-bit operands, ~2x the tensor
 *   work of DB200_SKETCH_SINGLE at l = 528.  What remains is the tensor cores' fp32 accumulation, which truncates
 *   toward zero: a sum over n points shrinks by ~2^-25 per accumulation step (1e-5 to 3e-5 relative at n = 4096 -
 *   8192).  The range finder of an SVM solve needs this product to match the FP64 path's dual objective to 1e-6:
 *   the single product's rounding of P shifts the sketched subspace enough to move the objective by ~4e-4 at
 *   n = 131072; the shrink does not matter there (the subspace is scale free).
 * DB200_SKETCH_COMPENSATED_PROMOTED: the compensated product with the accumulator restarted every 256 points j and
 *   each chunk added into Y in fp32 with round-to-nearest (reductions in L2), so the shrink is that of one chunk
 *   (~1e-6 relative).  ~1.8x the time of DB200_SKETCH_COMPENSATED at l = 528.
 * DB200_SKETCH_COMPENSATED_PROMOTED_COARSE: the same with chunks of 1024 points (~1.25x).
 * The mixed SVM path runs its range-finder passes coarse and its final pass (whose Y scales the core
 * C = Q^T K Q) with 256-point chunks: the dual objective then lies ~5e-7 from the FP64 path's at n = 4096 and
 * ~4e-7 at n = 131072 (with 1024-point chunks in the final pass too, 1.6e-6 at n = 4096; without promotion,
 * 6e-6 and 3e-6). */
#define DB200_SKETCH_SINGLE 0
#define DB200_SKETCH_P_SPLIT 1
#define DB200_SKETCH_COMPENSATED 2
#define DB200_SKETCH_COMPENSATED_PROMOTED 3
#define DB200_SKETCH_COMPENSATED_PROMOTED_COARSE 4

/* db200_rbf_sketch with a choice of sketch product (DB200_SKETCH_*).  Same arguments and layout otherwise. */
DB200_API int db200_rbf_sketch_ex(db200_context* ctx, int m, int n, int d, int l, const float* Xi, int ldxi,
                                  const float* Xj, int ldxj, int x_layout, const float* yi, const float* yj,
                                  const float* Omega, int ldo, float* Y, int ldy, float gamma, int product);

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
 * kernel over every block (the reference stops after the first, include/dkernel.h:43) and copies out; when A is
 * page-locked host memory the device can address (cudaMallocHost / cudaHostAlloc / registered), the kernel writes
 * it directly and no copy follows.  Synchronous.  Stands in for the rbf_kernel + tc_gemm host round trips of
 * include/dkernel.cu:132-231.
 */
DB200_API int db200_lra_host(db200_context* ctx, int n, int d, int k, const float* X, int ldx, const float* Y,
                             const float* O, int ldo, float* A, int lda, float gamma);

/* ------------------------------------------------------------------------------------------------------
 * Dense FP64 linear algebra on a 1 x 1 DMatrix (device pointers, column major).
 * ------------------------------------------------------------------------------------------------------ */

/* In-place upper Cholesky A = R^T R of the n x n matrix A (only the upper triangle is read; the strictly lower
 * part is zeroed), blocked right-looking with block size nb (<= 64; 0 = 64).  With nb = 64 and n <= 544 the whole
 * factor is one kernel on a thread-block cluster, in 32-column steps (the failing block named below is then the
 * 32-row block).  A non-positive pivot returns
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
  int precision;   /* DB200_MIXED (default) or DB200_FP64, see below */
  int refine_max;  /* iterative-refinement steps per Newton solve in DB200_MIXED (default 6) */
  int bias;        /* 0 (default): the reference's dual without a bias term.  1: the SVM with a bias, i.e. the
                      dual's equality constraint y^T a = 0 kept by every Newton step (a bordered Woodbury solve:
                      a second solve against y on the same capacity factor); the bias is reported in
                      db200_svm_report.b and replaces the estimate of include/dbarrier.h:420-442 */
} db200_barrier_params;

/* Precision of the path.
 * DB200_MIXED: kernel passes on the tensor cores, distances in split fp16 and the compensated sketch product with
 *   promoted fp32 accumulation (range finder DB200_SKETCH_COMPENSATED_PROMOTED_COARSE, final pass
 *   DB200_SKETCH_COMPENSATED_PROMOTED), which keeps the dual objective within ~5e-7 of the FP64 path's; the
 *   Woodbury capacity matrix
 *   I + Z^T D^-1 Z formed in integers on the int8 tensor cores from 8 signed 7-bit slices of every column (Ozaki
 *   scheme, error ~3e-14 of the column norms; from r = 2048 first 6 slices, ~3e-10, while refinement converges
 *   with them) and factored in FP64 while each Newton step refined
 *   against the exact FP64 operator (Z Z^T + D) reaches relative residual 1e-10, the FP64 capacity matrix after;
 *   objective, gradients, gap and line search in FP64.
 * DB200_FP64: plain FP64 everywhere (FP64 kernel blocks and products, FP64 capacity matrix): the comparator.
 * DB200_MIXED_FAST: DB200_MIXED with the single fp16 sketch product (DB200_SKETCH_SINGLE) in the kernel passes:
 *   half the tensor work of the compensated passes, dual objective ~4e-4 from the FP64 path's at n = 131072. */
#define DB200_MIXED 0
#define DB200_FP64 1
#define DB200_MIXED_FAST 2

/* What a solve did and where it ended. */
typedef struct db200_svm_report {
  double f;                /* dual objective f(a) = 0.5 a^T Z Z^T a - 1^T a at the returned a */
  double gap_barrier;      /* 2n/t / |f|: the barrier method's duality-gap bound */
  double gap_primal_dual;  /* (P(Z^T a, b) + f(a)) / |f|, P(w, b) = 0.5|w|^2 + C sum max(0, 1 - z_i.w - y_i b) */
  double t;                /* final barrier parameter */
  double nu;               /* shift of the Nystrom core Cholesky */
  int outer, newton;       /* barrier and Newton iterations */
  int status;              /* DB200_OK, DB200_ERR_MAXITER (caps reached) */
  int refine;              /* iterative-refinement steps taken (DB200_MIXED) */
  int fallbacks;           /* DB200_MIXED: 1 if a Newton step missed the refinement tolerance with the tensor-core
                              capacity matrix, after which the FP64 capacity matrix was used */
  double ms_sketch, ms_orth, ms_core, ms_barrier, ms_total;
  double b;                /* bias of the decision function sum_i a_i y_i K(x_i, x) + b (params.bias = 1, else 0):
                              the multiplier of y^T a = 0 at the last Newton step */
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
 * C = Q^T K Q; R^T R = C + nu I; Z = Q R^T.  K products use the fused kernel (db200_rbf_sketch) with
 * precision DB200_MIXED or the FP64 comparator (db200_rbf_sketch_f64) with DB200_FP64; orth is db200_cholqr2.
 * X point-major (ldx >= d), y and Omega (n x l, ldo >= n) device.  Synchronous. */
DB200_API int db200_lowrank(db200_context* ctx, int n, int d, int l, int q, const float* X, int ldx, const float* y,
                            const float* Omega, int ldo, float gamma, int precision, double* Z, int ldz,
                            db200_svm_report* rep);

/* The whole path: db200_lowrank followed by db200_svm_barrier (tests/testsvm.cpp:34-329 at one rank).
 * Outputs a (n, FP64) and Z (n x l FP64).  Synchronous; rep may be NULL. */
DB200_API int db200_svm_solve(db200_context* ctx, int n, int d, int l, int q, const float* X, int ldx,
                              const float* y, const float* Omega, int ldo, float gamma, double C,
                              const db200_barrier_params* p, double* a, double* Z, int ldz, db200_svm_report* rep);

/* ------------------------------------------------------------------------------------------------------
 * Row-sharded solve over several ranks (one process per GPU), the counterpart of DArray's row-distributed
 * matrices (include/darray.h:737-1054 replicates and reduces blocks over MPI).  Every rank holds all of X, y
 * and Omega and owns the rows [start, start + count) of Y = K Omega, of the factor Z and of the dual vector a
 * (db200_row_shard): the kernel passes need no exchange; CholeskyQR2 and the Nystrom core all-reduce one l x l
 * Gram each; the power and final passes need all of Q (gathered as a sum over ranks of zero-filled row blocks);
 * each Newton step all-reduces the r x r capacity matrix, the r-vectors Z^T x and a few scalars.  The library
 * calls the host-supplied collective for every exchange, so the plumbing (torch.distributed over NCCL, or a
 * test's in-process loopback) stays outside it.
 * ------------------------------------------------------------------------------------------------------ */
#define DB200_REDUCE_SUM 0
#define DB200_REDUCE_MAX 1
#define DB200_REDUCE_MIN 2
/* All-reduce of `count` FP64 values at device address buf in place (op: DB200_REDUCE_*), called with the
 * context's stream (cudaStream_t), on which buf is ready: the callee orders the reduction after the stream's
 * work and the stream's later work after the reduction (synchronising is enough), and returns 0 on success.
 * Every rank calls it with the same count and op in the same order. */
typedef int (*db200_allreduce_fn)(void* user, double* buf, long long count, int op, void* stream);
typedef struct db200_collective {
  int world;                   /* ranks sharing the problem */
  int rank;                    /* this rank, 0 <= rank < world */
  db200_allreduce_fn allreduce;
  void* user;                  /* passed back to allreduce */
} db200_collective;

/* Attach (c with world > 1) or detach (c == NULL or world == 1) a collective.  While one is attached:
 *   db200_lowrank and db200_svm_solve take the full X, y and Omega (n points) and write this rank's rows of Z
 *   (count x l, ldz >= count) and a (count) as db200_row_shard(n, world, rank) gives them;
 *   db200_svm_barrier takes this rank's rows: n = its row count, Z (n x r), y and a (n); the reports hold the
 *   global objective and gaps, the same on every rank.
 * db200_svm_solve_landmarks refuses to run (DB200_ERR_UNSUPPORTED); other entry points ignore it. */
DB200_API int db200_set_collective(db200_context* ctx, const db200_collective* c);

/* Contiguous balanced row blocks: rank k owns count = n / world (+1 for k < n % world) rows from start. */
DB200_API int db200_row_shard(int n, int world, int rank, int* start, int* count);

/* ------------------------------------------------------------------------------------------------------
 * Support for the one-rank DArray mirror (the headers under include/darray_b200/) and other host callers.
 * ------------------------------------------------------------------------------------------------------ */

/* Process-wide context on device 0 with its own stream (created on first use), the counterpart of the
 * reference's global handles set up by cuda_init() (include/dkernel.cu:12-17, 28-35). */
DB200_API db200_context* db200_default_context(void);
DB200_API int db200_release_default_context(void);

/* Device memory and stream-ordered copies on the context's stream (db200_copy_to_host also synchronizes). */
DB200_API int db200_malloc(db200_context* ctx, size_t bytes, void** ptr);
DB200_API int db200_free(db200_context* ctx, void* ptr);
DB200_API int db200_copy_to_device(db200_context* ctx, void* dst, const void* src, size_t bytes);
DB200_API int db200_copy_to_host(db200_context* ctx, void* dst, const void* src, size_t bytes);

/* C(m x n) = alpha op(A) op(B) + beta C, FP64, op in {N, T}; (T, T) is not provided.  Replaces
 * multiply_matrix<double> (include/cblas_like.h:51-60). */
DB200_API int db200_gemm(db200_context* ctx, char transA, char transB, int m, int n, int k, double alpha,
                         const double* A, int lda, const double* B, int ldb, double beta, double* C, int ldc);

/* C(m x n) = alpha op(A) B + beta C on FP32 data with FP64 accumulation, op(A) in {N, T} as in tc_sgemm
 * (include/dkernel.cu:234-275) and tc_gemm (:194-231, which ignored beta). */
DB200_API int db200_sgemm(db200_context* ctx, char transA, char transB, int m, int n, int k, float alpha,
                          const float* A, int lda, const float* B, int ldb, float beta, float* C, int ldc);

/* Singular values (descending) of the n x n matrix A, FP64 one-sided Jacobi; A is destroyed.  Replaces svd
 * (include/lapack_like.h:389-413), which returns only the singular values.  Synchronous. */
DB200_API int db200_svd_values(db200_context* ctx, int n, double* A, int lda, double* S);

/* Residual of a low-rank factor: out3 = {||K||_F, ||K - Z Z^T||_F, ratio} with K = diag(y) K(X, X) diag(y),
 * X point-major (ldx >= d), Z n x k FP64.  Replaces Knorm (include/dkernel.h:50-76), corrected to measure
 * K - Z Z^T and to accumulate over every block.  Synchronous. */
DB200_API int db200_knorm(db200_context* ctx, int n, int d, int k, const float* X, int ldx, const float* y,
                          const double* Z, int ldz, float gamma, double* out3);

/* x = (Z Z^T + diag(g))^-1 b by Sherman-Morrison-Woodbury with an FP64 Cholesky of I + Z^T g^-1 Z (Z n x r).
 * Solves the system pre_conjgrad (include/dbarrier.h:84-139) iterates on, exactly.  Synchronous. */
DB200_API int db200_woodbury_solve(db200_context* ctx, int n, int r, const double* Z, int ldz, const double* diag,
                                   const double* b, double* x);

/* Upper triangle of M(r x r) = Z^T diag(w) Z for Z n x r FP64 (w may be NULL = ones): the capacity-matrix
 * SYRK of the Woodbury Newton step (symmetric_update, include/cblas_like.h:62-69, with a row weight).
 * use_tensor_cores = 0: FP64 pipes (mma.sync f64); 1: tcgen05 kind::i8 on 8 signed 7-bit slices per value with
 * exact s32 sums (Ozaki scheme; error ~3e-14 ||z_p|| ||z_q||, z_p = column p of diag(sqrt(w)) Z); 5..8: that many
 * slices (error ~2e-8, 3e-10, 3e-12, 3e-14), products KS(KS + 1)/2 per 64-row chunk.
 * Stream-ordered. */
DB200_API int db200_gram_weighted(db200_context* ctx, int n, int r, const double* Z, int ldz, const double* w,
                                  double* M, int ldm, int use_tensor_cores);

/* Plain FP64 kernel x sketch (device pointers), the comparator of db200_rbf_sketch:
 *     Y(m x l, FP64) = diag(yi) K(Xi, Xj) diag(yj) Omega(n x l, FP64)
 * with FP64 norms, distances, exp and products in one fused launch on the FP64 tensor cores
 * (mma.sync.m16n8k8.f64): each CTA keeps 64 rows of Xi in shared memory and streams the points j, so K is never
 * stored.  Xi, Xj point-major float (ldxi, ldxj >= d), d <= 256.  Stream-ordered. */
DB200_API int db200_rbf_sketch_f64(db200_context* ctx, int m, int n, int d, int l, const float* Xi, int ldxi,
                                   const float* Xj, int ldxj, const float* yi, const float* yj, const double* Omega,
                                   int ldo, double* Y, int ldy, double gamma);

/* Materialised FP64 RBF block K(m x n) = diag(yi) exp(-gamma D2(Xi, Xj)) diag(yj), column major (ldk >= m):
 * FP64 norms, an FP64 tensor-core Gram for the cross term, FP64 exp.  The FP64 counterpart of db200_rbf_block
 * (include/dkernel.cu:132-190).  Xi, Xj point-major float.  Stream-ordered. */
DB200_API int db200_rbf_block_f64(db200_context* ctx, int m, int n, int d, const float* Xi, int ldxi, const float* Xj,
                                  int ldxj, const float* yi, const float* yj, double* K, int ldk, double gamma);

/* y = alpha x + beta y + gamma elementwise on n FP64 device values (x may be NULL): the vector updates of
 * include/dbarrier.h:60-73 (Grad = Grad_f + Grad_Phi) and of the D + n I shift of pre_conjgrad. */
DB200_API int db200_vec_update(db200_context* ctx, int n, double alpha, const double* x, double beta, double* y,
                               double gamma);

/* The barrier terms at a (device vectors of length n, any output may be NULL): gradf = Z Z^T a - 1 (Grad_f),
 * gradphi = (-1/a + 1/(C-a))/t (Grad_Phi), grad = gradf + gradphi (Grad), D = (1/a^2 + 1/(C-a)^2)/t (Hess_Phi),
 * and on the host f_gg[0] = f(a) = 0.5 a^T Z Z^T a - 1^T a (f), f_gg[1] = f(a) - sum(log a + log(C-a))/t (gg).
 * include/dbarrier.h:14-81.  Synchronous. */
DB200_API int db200_barrier_terms(db200_context* ctx, int n, int k, const double* Z, int ldz, const double* a,
                                  double C, double t, double* gradf, double* gradphi, double* grad, double* D,
                                  double* f_gg);

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
 * Every call resolves the array's device address in the current context (cudaGetSymbolAddress, with the
 * stream's device current), so the address is never stale after a device reset or in a caller's own context;
 * the first call on a device also loads the library's device code into that context, so make the first call
 * before any stream capture begins.  n = 0 writes Y = 0, as db200_rbf_sketch does.  All calls share the one
 * array and it keeps the previous call's contents (every byte a call reads is written by that call first);
 * calls that overlap on the GPU -- from two host threads, or on two streams -- race on it and must be serialised
 * by the caller.
 */
#define DB200_NOALLOC_SCRATCH_BYTES (32u << 20)
DB200_API int db200_rbf_sketch_noalloc(void* stream, int m, int n, int d, int l, const float* Xi, int ldxi,
                                       const float* Xj, int ldxj, int x_layout, const float* yi, const float* yj,
                                       const float* Omega, int ldo, float* Y, int ldy, float gamma);

/* ------------------------------------------------------------------------------------------------------------
 * Batched instances: many independent problems of uneven n, d, l, gamma and C (hyperparameter grids, one-vs-rest
 * classes) in one persistent launch of the tile engine.  The reference runs one problem per process
 * (tests/testsvm.cpp:34-329); these entry points have no counterpart there.
 * ------------------------------------------------------------------------------------------------------------ */

/* One sketch problem Y (m x l) = diag(yi) K(Xi, Xj) diag(yj) Omega (n x l), as db200_rbf_sketch, plus an optional
 * tile plan: n_panels sketch panels of `panel` columns (a multiple of 16, <= 320) with g_bufs (1 or 2) distance
 * buffers in tensor memory, panel + 64 + 128 g_bufs <= 512; n_panels = 0 selects the default plan. */
typedef struct {
  int m, n, d, l;
  const float* Xi;
  int ldxi;
  const float* Xj;
  int ldxj;
  const float* yi;
  const float* yj;
  const float* Omega;
  int ldo;
  float* Y;
  int ldy;
  float gamma;
  int n_panels, panel, g_bufs;
} db200_sketch_job;

/* Every job's K.Omega in one persistent launch (work items of all jobs interleaved over the CTA pairs).  Device
 * pointers, point-major points.  Stream-ordered. */
DB200_API int db200_rbf_sketch_batched(db200_context* ctx, int count, const db200_sketch_job* jobs);

/* One SVM instance of db200_svm_solve_batched (device pointers). */
typedef struct {
  int n, d, l;           /* points, features, sketch width */
  const float* X;        /* point-major, ldx >= d */
  int ldx;
  const float* y;        /* labels +-1 */
  float gamma;
  double C;
  const float* Omega;    /* n x l Gaussian test matrix, column major */
  int ldo;
  double* Z;             /* out: n x l FP64 factor, diag(y) K diag(y) ~ Z Z^T */
  int ldz;
  double* a;             /* out: n dual variables */
  int n_panels, panel, g_bufs;  /* tile plan of the sketch passes; n_panels = 0: default */
} db200_svm_instance;

typedef struct {
  double ms_pack, ms_sketch, ms_orth, ms_core, ms_barrier, ms_total;
  int kernel_passes;     /* persistent launches over all instances */
  int graph_replays;     /* of those, replays of a captured CUDA graph (test-matrix packing + tile launch) */
  int workers;           /* host threads (each with its own context and stream) running the barriers */
} db200_batch_report;

/* Mixed-precision SVM solves of `count` instances: the q + 2 kernel passes of every instance run as single
 * persistent launches over all instances (after the first, replayed from a captured CUDA graph when use_graph),
 * CholeskyQR2 and the Nystrom core per instance in FP64, then the barrier of each instance
 * (db200_svm_barrier with `params`) on `workers` host threads with their own contexts and streams.  reports: count
 * entries (barrier results per instance).  Returns the first failing instance's status.  Synchronous. */
DB200_API int db200_svm_solve_batched(db200_context* ctx, int count, const db200_svm_instance* inst, int q,
                                      const db200_barrier_params* params, int use_graph, int workers,
                                      db200_svm_report* reports, db200_batch_report* brep);

/* ------------------------------------------------------------------------------------------------------------
 * Learned Nystrom landmarks.  No counterpart in the reference, which always sketches with a Gaussian Omega
 * (include/dkernel.h:13-46, tests/testsvm.cpp:94-134): a small MLP predicts per-point ridge leverage scores, r
 * landmarks are drawn by those scores, and the factor Z = K(:, L) chol(K(L, L))^-1 replaces the Gaussian sketch
 * when a sampled residual estimate meets the tolerance; otherwise the Gaussian pipeline (db200_lowrank) runs.
 * All pointers are device pointers; points are point-major float (ldx >= d).
 * ------------------------------------------------------------------------------------------------------------ */

/* Distance from each of the n points to its k-th nearest neighbour among the s reference points ref_idx
 * (indices into X; a point is never its own neighbour).  k <= 16.  out: n floats.  Stream-ordered. */
DB200_API int db200_knn_distance(db200_context* ctx, int n, int d, const float* X, int ldx, int s, const int* ref_idx,
                                 int k, float* out);

/* Leverage-model inputs, row-major n x (d + 2): [x_i, ||x_i||, knn_i].  Stream-ordered. */
DB200_API int db200_leverage_features(db200_context* ctx, int n, int d, const float* X, int ldx, const float* knn,
                                      float* F);

/* Ridge leverage scores of K ~ Z Z^T (Z n x r FP64): lev_i = z_i^T (Z^T Z + lambda I)^-1 z_i, in FP64 (Gram,
 * Cholesky, triangular inverse, row sums of squares).  Synchronous. */
DB200_API int db200_ridge_leverage(db200_context* ctx, int n, int r, const double* Z, int ldz, double lambda,
                                   double* lev);

/* The leverage MLP: in_dim inputs (standardised with a per-input mean and scale), `hidden` ReLU layers of `width`
 * units, one linear output.  Weights and activations are bf16 in the forward pass, accumulation fp32; master
 * weights, gradients and Adam moments fp32.  Flat parameter order: for each layer l, W_l (out x in, row major)
 * then b_l. */
typedef struct db200_mlp db200_mlp;
DB200_API int db200_mlp_create(db200_context* ctx, int in_dim, int width, int hidden, unsigned long long seed,
                               db200_mlp** out);
DB200_API void db200_mlp_destroy(db200_mlp* net);
DB200_API int db200_mlp_param_count(const db200_mlp* net);
/* Copy the fp32 master parameters to / from host memory (param_count floats). */
DB200_API int db200_mlp_get_params(db200_context* ctx, const db200_mlp* net, float* host);
DB200_API int db200_mlp_set_params(db200_context* ctx, db200_mlp* net, const float* host);
/* Input standardisation: x' = (x - mean) * scale (host arrays of in_dim floats). */
DB200_API int db200_mlp_set_input_scaling(db200_context* ctx, db200_mlp* net, const float* mean, const float* scale);
/* out[i] = net(F[i, :]) for m rows of F (device, row-major m x in_dim).  Stream-ordered. */
DB200_API int db200_mlp_forward(db200_context* ctx, const db200_mlp* net, int m, const float* F, float* out);
/* Loss 0.5 mean_i (net(F_i) - t_i)^2 and its gradient with respect to the flat parameters (device array of
 * param_count floats).  loss: host.  Synchronous. */
DB200_API int db200_mlp_gradients(db200_context* ctx, db200_mlp* net, int m, const float* F, const float* target,
                                  float* loss, float* grads);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the loss above; loss (host, may be NULL). */
DB200_API int db200_mlp_adam_step(db200_context* ctx, db200_mlp* net, int m, const float* F, const float* target,
                                  float lr, float* loss);

/* Gumbel keys for sampling without replacement proportional to exp(logits): keys_i = logits_i + G_i, G_i a
 * seeded standard Gumbel variate; the k largest keys are a weighted sample (Gumbel top-k).  Stream-ordered. */
DB200_API int db200_gumbel_keys(db200_context* ctx, int n, const float* logits, unsigned long long seed, float* keys);
/* Indices of the k largest keys (any order).  Synchronous. */
DB200_API int db200_select_topk(db200_context* ctx, int n, const float* keys, int k, int* idx);

/* Nystrom factor on landmarks idx (r indices): C = diag(y) K(:, L) diag(y_L) (n x r, fused tile kernel),
 * W = C(L, :) in FP64, R^T R = W + nu I (shifted Cholesky, nu = 1e-7 tr(W)/r, x10 until positive definite),
 * Z = C R^-1 (n x r FP64), so diag(y) K diag(y) ~ Z Z^T.  nu_out: host, may be NULL.  Synchronous. */
DB200_API int db200_landmark_factor(db200_context* ctx, int n, int d, const float* X, int ldx, const float* y,
                                    float gamma, int r, const int* idx, double* Z, int ldz, double* nu_out);
/* db200_landmark_factor with C = diag(y) K(:, L) diag(y_L) in a chosen precision: DB200_MIXED (or
 * DB200_MIXED_FAST): the tcgen05 tile engine's fp32 kernel block; DB200_FP64: the FP64 kernel block
 * (db200_rbf_block_f64), the comparator.  Synchronous. */
DB200_API int db200_landmark_factor_ex(db200_context* ctx, int n, int d, const float* X, int ldx, const float* y,
                                       float gamma, int r, const int* idx, double* Z, int ldz, double* nu_out,
                                       int precision);

/* Sampled residual ||Q(:, S) - Z Z(S, :)^T||_F / ||Q(:, S)||_F with Q = diag(y) K diag(y) over s columns S
 * (indices): an estimate of ||Q - Z Z^T||_F / ||Q||_F.  est: host.  Synchronous. */
DB200_API int db200_residual_estimate(db200_context* ctx, int n, int d, const float* X, int ldx, const float* y,
                                      float gamma, int r, const double* Z, int ldz, int s, const int* sample_idx,
                                      double* est);

typedef struct {
  int used_fallback;     /* 1 when the Gaussian sketch replaced the landmark factor */
  int rank;              /* columns of Z actually used by the barrier */
  double residual_est;   /* sampled residual of the landmark factor */
  double residual_fallback; /* sampled residual of the Gaussian factor (fallback only, else 0) */
  double ms_features, ms_predict, ms_select, ms_factor, ms_residual, ms_fallback;
} db200_landmark_report;

/* The landmark selection of db200_svm_solve_landmarks on its own: features (8-NN distance over s_knn reference
 * points drawn with `seed`) -> MLP log-leverage -> Gumbel keys (`seed`) -> the r largest, written to idx (device,
 * r ints).  The same seed gives the same landmarks as the solve.  Synchronous. */
DB200_API int db200_select_landmarks(db200_context* ctx, int n, int d, int r, const float* X, int ldx,
                                     const db200_mlp* net, unsigned long long seed, int s_knn, int* idx);

/* Learned-landmark SVM solve: features (8-NN distance over s_knn reference points) -> MLP log-leverage ->
 * Gumbel top-r landmarks -> Nystrom factor -> sampled residual estimate (s_res columns); if the estimate exceeds
 * tol the Gaussian pipeline db200_lowrank(l_fb = Omega's columns, q) builds the factor instead; then the barrier
 * (db200_svm_barrier) on the factor.  The landmark columns K(:, L) (n r d work, r / n of one kernel pass) are FP64
 * (db200_landmark_factor_ex with DB200_FP64) unless params->precision is DB200_MIXED_FAST, which takes the tile
 * engine's fp32 block.  Z: n x max(r, l_fb) FP64, a: n.  Synchronous. */
DB200_API int db200_svm_solve_landmarks(db200_context* ctx, int n, int d, int r, const float* X, int ldx,
                                        const float* y, float gamma, double C, const db200_mlp* net,
                                        unsigned long long seed, int s_knn, int s_res, double tol,
                                        const float* Omega, int ldo, int l_fb, int q,
                                        const db200_barrier_params* params, double* a, double* Z, int ldz,
                                        db200_svm_report* rep, db200_landmark_report* lrep);

/* LU factorisation of the m x n FP32 matrix A (device, column major, lda >= m) in place: A = P L U with L unit
 * lower (below the diagonal) and U upper, blocked right-looking with panels of 32 columns.  Replaces
 * lu_factorize_partial_pivot (include/lapack_like.h:179-219, the unblocked panel of :220-279),
 * lu_factorize_partial_pivot_replicate_panel (:134-177) and lu_factorize_no_pivot (:93-131):
 *   pivot = 1: partial pivoting, the pivot of column j the row of largest |a| at or below j (the first such row on
 *     ties, as the reference's scan); ipiv[j] (device, min(m, n) ints) = 1-based pivot row relative to A's first
 *     row, as LAPACK and the reference record it;
 *   pivot = 0: no interchanges (ipiv[j] = j + 1).
 *   swap_left_panels = 1: every panel's interchanges also reach the columns of earlier panels and the nleft
 *     columns that precede A in memory (A - nleft*lda ...), as lu_factorize_partial_pivot permutes the rows left
 *     of the factored block (:212); 0: only the columns right of the panel, as the replicate_panel variant (:162).
 * A zero pivot returns DB200_ERR_SINGULAR naming its column (the reference asserts).  Synchronous. */
DB200_API int db200_lu_factorize(db200_context* ctx, int m, int n, int nleft, float* A, int lda, int* ipiv,
                                 int pivot, int swap_left_panels);

/* ------------------------------------------------------------------ LIBSVM text input */
#define DB200_F32 0 /* float X and y */
#define DB200_F64 1 /* double X and y */

/* Parse the first n lines of LIBSVM text ("label index:value index:value ...", lines ended by '\n') held in
 * device memory (`bytes` characters at `text`, any alignment) into device X and y, as read_input_file<T>
 * (include/read_input.h:8-36) does on the host:
 *   - tokens are separated by ' ' only (runs of blanks collapse); the first token of a line is the label and
 *     y[i] = +1 when it converts (strtod, then to T) to exactly 1, else -1;
 *   - every further token is "index:value": index = atoi of the part before the first ':', value = strtod of the
 *     part after it (of the whole token when it has no ':'); X[(index - 1) + i*ldx] = value for index >= 1,
 *     tokens with index < 1 are skipped; repeated indices keep the last value;
 *   - values are correctly rounded to double and then, for DB200_F32, to float, so results are bit-identical to
 *     the reference's; "inf", "infinity" and "nan" are accepted;
 *   - entries of X and y that the text does not name keep their values.
 * The reference indexes rows with stride d and ignores ldx; here the stride is ldx (>= d), the same at its call
 * site (tests/testsvm.cpp:71, ldx = d).  lines_out (host, may be NULL) receives the lines parsed: min(n, lines in
 * the text).  Where the reference's behaviour is undefined or would differ, the call fails instead, naming the
 * first offending line in db200_last_error: DB200_ERR_INVALID for a feature index above d (the reference writes
 * past the row) and for a last line of blanks only (the reference passes NULL to atof); DB200_ERR_UNSUPPORTED for
 * hexadecimal values, "nan(...)" payloads, values with more than 38 significant digits and NUL bytes.
 * dtype: DB200_F32 or DB200_F64.  Synchronous. */
DB200_API int db200_libsvm_parse(db200_context* ctx, const char* text, long long bytes, int n, int d, int dtype,
                                 void* X, long long ldx, void* y, int* lines_out);

/* read_input_file<T>(filename, n, d, X, ldx, Y) (include/read_input.h:8-36) with HOST X and y: the file is read
 * in 32 MiB pieces through pinned staging, each piece's copy to the device overlapping the next read, parsed by
 * db200_libsvm_parse and X, y copied back (X and y are copied to the device first, so entries the file does not
 * name keep their values).  A file that cannot be opened returns DB200_ERR_INVALID (the reference exits).
 * Synchronous. */
DB200_API int db200_read_libsvm(db200_context* ctx, const char* path, int n, int d, int dtype, void* X,
                                long long ldx, void* y, int* lines_out);

#ifdef __cplusplus
}
#endif

#endif /* DARRAY_B200_H */
