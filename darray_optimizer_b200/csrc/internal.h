// Internal host-side interfaces shared by the .cu translation units of libdarray_b200.
#pragma once
#include <cstddef>
#include <cstdint>
#include <functional>
#include <string>
#include <utility>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/darray_b200.h"

struct db200_context {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int* d_status = nullptr;       // [0] device status word written by kernels whose bounded waits give up,
                                 // [1] arrival counter of potrf_block_kernel (zero between launches)
  void* ws = nullptr;            // device workspace (packed operands, small factors)
  size_t ws_size = 0;
  void* io = nullptr;            // device staging for the host-pointer entry points
  size_t io_size = 0;
  // Further grow-only device buffers, one per call level so nested calls never share one:
  // [0] dense linear algebra internals, [1] low-rank / solve pipeline, [2] barrier solver, [3] spare,
  // [4] learned-landmark pipeline (features, scores, landmark indices).
  void* slot[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  size_t slot_size[5] = {0, 0, 0, 0, 0};
  double* h_pinned = nullptr;    // small pinned host staging area for scalar readbacks
  void* h_stage = nullptr;       // pinned host staging for file input (two halves, grow-only)
  size_t h_stage_size = 0;
  void* tile_table = nullptr;    // instance table of the tile engine (grow-only)
  size_t tile_table_size = 0;
  // Worker contexts (own stream and buffers each) of the batched solve, kept across calls so their buffers stay
  // grown and no call pays context creation.
  std::vector<db200_context*> workers;
  std::string last_error;
  long long launches = 0;        // kernels launched through this context
  // Optional per-launch timing of the tcgen05 tile kernels (CUDA events on the launching stream).
  bool profiling = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;
  // CUDA graphs of repeated launch sequences (the barrier's capacity-matrix factor), keyed by the pointers and
  // sizes they were captured with; captured on a private non-blocking stream and replayed on `stream`.
  struct GraphEntry {
    std::vector<long long> key;
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;  // kernels in the graph (added to `launches` per replay)
  };
  cudaStream_t cap_stream = nullptr;
  std::vector<GraphEntry> graphs;
  bool graphs_off = false;   // a capture failed once: sequences run eagerly from then on
  // Row-sharded solves (db200_set_collective): the host's all-reduce; world 1 = none attached.
  int coll_world = 1, coll_rank = 0;
  // Largest thread-block cluster of the one-launch Cholesky (potrf_cluster.cu) this device holds; 0: none.
  int potrf_nc_max = 0;
  db200_allreduce_fn coll_fn = nullptr;
  void* coll_user = nullptr;
};

namespace db200 {

// Error helpers: set ctx->last_error and return the status.
int fail(db200_context* ctx, int status, const std::string& msg);
int cuda_fail(db200_context* ctx, cudaError_t err, const char* what);

#define DB200_CUDA(ctx, call)                                   \
  do {                                                          \
    cudaError_t e_ = (call);                                    \
    if (e_ != cudaSuccess) return ::db200::cuda_fail((ctx), e_, #call); \
  } while (0)

// Launch accounting and optional event timing around the dominant (tile) kernels.
inline void count_launch(db200_context* ctx, int k = 1) { ctx->launches += k; }
void prof_begin(db200_context* ctx, cudaEvent_t* e0);
void prof_end(db200_context* ctx, cudaEvent_t e0);

// Grow-only workspace; returns nullptr on failure (ctx->last_error set).
void* workspace(db200_context* ctx, size_t bytes);
void* io_buffer(db200_context* ctx, size_t bytes);
enum { SLOT_LA = 0, SLOT_PIPE = 1, SLOT_BAR = 2, SLOT_SPARE = 3, SLOT_LAND = 4 };
void* slot_buffer(db200_context* ctx, int slot, size_t bytes);

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
inline int round_up(int x, int a) { return (x + a - 1) / a * a; }

// Bump allocator over one workspace request.
struct Carve {
  char* base;
  size_t off = 0;
  template <class T>
  T* take(size_t count) {
    off = align_up(off, 256);
    T* p = reinterpret_cast<T*>(base + off);
    off += count * sizeof(T);
    return p;
  }
};

// ------------------------------------------------------------------ LU (lu.cu)
int lu_factorize(db200_context* ctx, int m, int n, int nleft, float* A, long long lda, int* ipiv, int pivot,
                 int swap_left_panels);

// ------------------------------------------------------------------ RBF tile engine (rbf_tile.cu)
// SKETCH: Y = (y_i y_j exp(-gamma d_ij^2)) Omega; KBLOCK: K = y_i y_j exp(-gamma d_ij^2) stored; UPDATE: the distance
// GEMM alone, out[i, j] += alpha x_i.x_j (TileJob::gamma carries alpha), the split-fp16 product of a rank-d update;
// KNN: the 8 smallest squared distances d_ij^2 of each point i over the points j of each quarter of the tile columns,
// sorted, in out[32 i + 8 quarter + t] (TileJob::gamma = 1; TileJob::yj carries the points' indices as int, and j
// with index i is skipped)
enum RbfMode { RBF_MODE_SKETCH = 0, RBF_MODE_KBLOCK = 1, RBF_MODE_UPDATE = 2, RBF_MODE_KNN = 3 };

struct PackedPoints {
  const void* xp = nullptr;   // fp16 [npad][2*dp]: [hi | lo] split of each point scaled by the set's 2^e
  const float* norms = nullptr;  // fp32: ||x||^2 [npad] (zero on padding rows), then max |x| bits and 2^-e
  int n = 0, npad = 0, dp = 0;
  // a slice of a packed set (rows from a multiple of 128, npad a multiple of 128): the parent's norms + npad, where
  // its max |x|, scale and lo flag sit; null for a set of its own
  const float* tail = nullptr;
};
// floats of the norms-and-scale array of a packed set of npad points
inline size_t packed_norm_floats(int npad) { return (size_t)npad + 64; }

// Pack points into the split-fp16 operand layout (one power-of-two scale for the set) plus squared norms and the
// scale (norms must hold packed_norm_floats(npad) floats).  Two kernels: the set's max |x|, then the split.
// layout: DB200_POINT_MAJOR (x_ik = X[k + i*ldx]) or DB200_FEATURE_MAJOR (x_ik = X[i + k*ldx]).
int pack_points(db200_context* ctx, const float* X, int ldx, int layout, int n, int d, int dp, int npad, void* xp,
                float* norms);

// Omega^T (fp16, [lrows][njpad]) with the column labels folded in: Op[c][j] = y_j * Omega[j + c*ldo]; with
// comp = 2 a second [lrows][njpad] block follows with the lo parts (fp16 of the hi rounding's residual).
int pack_sketch(db200_context* ctx, const float* Omega, int ldo, const float* yj, int n, int l, int njpad, int lrows,
                void* op, int comp = 0);

// comp: sketch product P.Om (0), + P_lo.Om (1), + P_hi.Om_lo (2, compensated); promote: j tiles per TMEM
// accumulation chunk, each chunk added into Y in fp32 (0: one accumulation over all j)
struct SketchPlan {
  int n_panels = 1, panel = 16, lrows = 16, g_bufs = 2, comp = 0, promote = 0;
};
SketchPlan plan_sketch(int l, int comp = 0);
// halves (2-byte elements) of the packed Omega~ operand for a plan over njpad points
inline size_t packed_sketch_halves(const SketchPlan& p, int njpad) {
  return (size_t)p.lrows * njpad * (p.comp == 2 ? 2 : 1);
}
int feature_pad(int d);  // dp: padded feature count of the split operand
// Packed point counts are padded to whole 256-row tiles (one CTA pair of the tile kernel), on both sides, so that
// a set used as rows and as columns packs once.
inline int point_pad(int n) { return round_up(n < 1 ? 1 : n, 256); }

// One problem of the fused tile engine: Y = diag(yi) K(Xi, Xj) diag(yj) Omega (SKETCH, `op` = packed Omega^T) or
// the kernel block (KBLOCK), written to `out` (column major, leading dimension ldo).
struct TileJob {
  PackedPoints pi, pj;
  const float* yi = nullptr;
  const float* yj = nullptr;
  const void* op = nullptr;
  SketchPlan plan;
  int om_lo = 0;  // comp = 2: row offset of the lo rows of Omega~ from `op`
  int l = 0;
  float gamma = 0.f;
  float* out = nullptr;
  long long ldo = 0;
};
// A prepared launch: the instance table is on the device; launch_rbf_plan only launches (graph-capturable).
struct TilePlan {
  int mode = 0, count = 0, n_items = 0, nsx = 0, nso = 0, nkc_max = 0, panel_max = 0, om_mult = 1;
  int clusters = 0;  // persistent grid: CTA pairs resident at once (at most one per item)
  bool lean = false; // SKETCH with the single product and no promotion in every instance: the lean kernel
  size_t smem = 0;
  const void* table = nullptr;
  alignas(64) unsigned char tm1[4 * 128];  // instance 0's tensor maps (kernel parameters of one-instance launches)
};
size_t tile_table_bytes(int count);
// Build the instance table of `count` jobs and copy it to the device (table_storage if given, else a context
// buffer).  Stream-ordered.
int prepare_rbf_tiles(db200_context* ctx, int mode, const TileJob* jobs, int count, void* table_storage,
                      size_t table_capacity, TilePlan* plan);
// One persistent launch over every work item of the prepared jobs.
int launch_rbf_plan(db200_context* ctx, const TilePlan& plan);

// ------------------------------------------------------------------ SVM pipeline pieces (svm.cpp)
// Orthonormalise Y (n x l, FP64) in place by CholeskyQR2 (shifted CholeskyQR3 when the Gram is not positive
// definite); R (l x l) optional.  tc_gram: Grams on the int8 tensor cores (Ozaki, 8 digits), else FP64 pipes.
// dist: Y holds this rank's rows of a row-sharded matrix and the Grams are all-reduced over the attached collective.
int cholqr2_impl(db200_context* ctx, int n, int l, double* Y, int ldy, double* Rout, int ldr, bool tc_gram,
                 bool dist = false);
// Nystrom core: C = Q^T Yk (Yk = K Q), symmetrised; R^T R = C + nu I (shifted Cholesky); Z = Q R^T.  dist: Q, Yk
// and Z are this rank's rows and C is all-reduced.
template <typename TY>
int nystrom_core(db200_context* ctx, int n, int l, const double* Q, const TY* Yk, double* Cm, double* R, int* d_pair,
                 double* d_scalar, double* Z, int ldz, double* nu_out, bool dist = false);
// The log-barrier solve of db200_svm_barrier.  dist: Z, y and a are this rank's n rows of a row-sharded problem and
// every reduction over rows goes through the attached collective.
int svm_barrier_impl(db200_context* ctx, int n, int r, const double* Z, int ldz, const float* y, double C,
                     const db200_barrier_params& P, double* a, db200_svm_report* rep, bool dist = false);

// Bytes of the context buffers cholqr2_impl (SLOT_LA) and svm_barrier_impl (SLOT_BAR, mixed: with the int8 Gram's
// scratch) take for n rows and l (r) columns; callers that run many problems on one context can size them up front.
size_t cholqr2_slot_bytes(int n, int l);
size_t barrier_slot_bytes(int n, int r, bool mixed);

// Row-sharded solves: whether a collective of more than one rank is attached, and its all-reduce of `count` FP64
// values at device address buf (in place, on the context's stream; a no-op when none is attached).
inline bool sharded(const db200_context* ctx) { return ctx->coll_world > 1 && ctx->coll_fn; }

// Enqueue what `body` launches on ctx->stream through a CUDA graph cached under `key` (the sequence's pointers and
// sizes): the first call with a key captures body on a private stream and instantiates it, later calls replay
// it with one launch.  body must only enqueue work on ctx->stream (no host synchronisation or reads).  If a
// capture fails, the context runs every sequence eagerly from then on.
int graph_run(db200_context* ctx, const std::vector<long long>& key, const std::function<int()>& body);
int allreduce(db200_context* ctx, double* buf, long long count, int op);

// Launch the fused tile kernel for one problem.  For RBF_MODE_SKETCH, `op` is the packed Omega^T and `out` is Y
// (m x l, column major, leading dimension ldo); for RBF_MODE_KBLOCK, `out` is the kernel block K (m x n, column
// major).  table_storage: device memory for the one-instance table (NULL: a context buffer).
int launch_rbf_tiles(db200_context* ctx, int mode, const PackedPoints& pi, const PackedPoints& pj, const float* yi,
                     const float* yj, const void* op, const SketchPlan& plan, int l, float gamma, float* out,
                     int ldo, void* table_storage = nullptr, size_t table_capacity = 0);

// Per-panel instances of exact widths for a multi-panel sketch job (plan.n_panels panels covering roundup(l, 16)),
// appended to `out`; a one-panel job is appended as it is.
void exact_panel_jobs(const TileJob& base, std::vector<TileJob>& out);
// The sketch as one launch over per-panel instances of exact widths (plan.n_panels panels covering roundup(l, 16)).
int launch_rbf_sketch_exact(db200_context* ctx, const PackedPoints& pi, const PackedPoints& pj, const float* yi,
                            const void* op, const SketchPlan& plan, int l, float gamma, float* out, int ldo);

}  // namespace db200
