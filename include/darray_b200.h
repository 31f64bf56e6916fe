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
