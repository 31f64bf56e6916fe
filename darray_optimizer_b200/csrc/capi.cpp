// C ABI of libdarray_b200: context management and the RBF kernel / sketch entry points.
#include <cstdio>
#include <cstring>
#include <atomic>
#include <string>

#include "internal.h"
#include "la64.h"

namespace db200 {

int fail(db200_context* ctx, int status, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return status;
}

int cuda_fail(db200_context* ctx, cudaError_t err, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(err);
  return fail(ctx, err == cudaErrorMemoryAllocation ? DB200_ERR_NOMEM : DB200_ERR_CUDA, m);
}

void* workspace(db200_context* ctx, size_t bytes) {
  if (bytes <= ctx->ws_size) return ctx->ws;
  // Growing: queued work may still read the old buffer.
  cudaStreamSynchronize(ctx->stream);
  if (ctx->ws) cudaFree(ctx->ws);
  ctx->ws = nullptr;
  ctx->ws_size = 0;
  size_t want = align_up(bytes + bytes / 8, 1 << 20);
  cudaError_t e = cudaMalloc(&ctx->ws, want);
  if (e != cudaSuccess) {
    ctx->ws = nullptr;
    cuda_fail(ctx, e, "cudaMalloc(workspace)");
    return nullptr;
  }
  ctx->ws_size = want;
  return ctx->ws;
}

void prof_begin(db200_context* ctx, cudaEvent_t* e0) {
  *e0 = nullptr;
  if (!ctx->profiling) return;
  if (cudaEventCreate(e0) != cudaSuccess || cudaEventRecord(*e0, ctx->stream) != cudaSuccess) *e0 = nullptr;
}

void prof_end(db200_context* ctx, cudaEvent_t e0) {
  if (!ctx->profiling || !e0) return;
  cudaEvent_t e1;
  if (cudaEventCreate(&e1) != cudaSuccess) return;
  cudaEventRecord(e1, ctx->stream);
  ctx->prof_events.emplace_back(e0, e1);
}

static void prof_clear(db200_context* ctx) {
  for (auto& p : ctx->prof_events) {
    cudaEventDestroy(p.first);
    cudaEventDestroy(p.second);
  }
  ctx->prof_events.clear();
}

void* io_buffer(db200_context* ctx, size_t bytes) {
  if (bytes <= ctx->io_size) return ctx->io;
  cudaStreamSynchronize(ctx->stream);
  if (ctx->io) cudaFree(ctx->io);
  ctx->io = nullptr;
  ctx->io_size = 0;
  size_t want = align_up(bytes, 1 << 20);
  cudaError_t e = cudaMalloc(&ctx->io, want);
  if (e != cudaSuccess) {
    ctx->io = nullptr;
    cuda_fail(ctx, e, "cudaMalloc(io buffer)");
    return nullptr;
  }
  ctx->io_size = want;
  return ctx->io;
}

void* slot_buffer(db200_context* ctx, int slot, size_t bytes) {
  if (bytes <= ctx->slot_size[slot]) return ctx->slot[slot];
  cudaStreamSynchronize(ctx->stream);
  if (ctx->slot[slot]) cudaFree(ctx->slot[slot]);
  ctx->slot[slot] = nullptr;
  ctx->slot_size[slot] = 0;
  size_t want = align_up(bytes, 1 << 20);
  cudaError_t e = cudaMalloc(&ctx->slot[slot], want);
  if (e != cudaSuccess) {
    ctx->slot[slot] = nullptr;
    cuda_fail(ctx, e, "cudaMalloc(slot buffer)");
    return nullptr;
  }
  ctx->slot_size[slot] = want;
  return ctx->slot[slot];
}

int graph_run(db200_context* ctx, const std::vector<long long>& key, const std::function<int()>& body) {
  if (ctx->graphs_off) return body();
  for (auto& e : ctx->graphs) {
    if (e.key != key) continue;
    DB200_CUDA(ctx, cudaGraphLaunch(e.exec, ctx->stream));
    ctx->launches += e.launches;
    return DB200_OK;
  }
  if (!ctx->cap_stream && cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    ctx->graphs_off = true;
    return body();
  }
  const long long launches0 = ctx->launches;
  cudaStream_t saved = ctx->stream;
  ctx->stream = ctx->cap_stream;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal);
  int st = (e == cudaSuccess) ? body() : DB200_ERR_CUDA;
  if (e == cudaSuccess) e = cudaStreamEndCapture(ctx->cap_stream, &g);
  ctx->stream = saved;
  cudaGraphExec_t x = nullptr;
  if (e == cudaSuccess && st == DB200_OK && g) e = cudaGraphInstantiate(&x, g, 0);
  if (g) cudaGraphDestroy(g);
  const long long captured = ctx->launches - launches0;
  ctx->launches = launches0;
  if (e != cudaSuccess || st != DB200_OK || !x) {
    cudaGetLastError();  // the failed capture's error is not the caller's
    ctx->graphs_off = true;
    return body();
  }
  if (ctx->graphs.size() >= 64) {
    cudaGraphExecDestroy(ctx->graphs.front().exec);
    ctx->graphs.erase(ctx->graphs.begin());
  }
  ctx->graphs.push_back({key, x, captured});
  DB200_CUDA(ctx, cudaGraphLaunch(x, ctx->stream));
  ctx->launches += captured;
  return DB200_OK;
}

int allreduce(db200_context* ctx, double* buf, long long count, int op) {
  if (!sharded(ctx) || count <= 0) return DB200_OK;
  const int st = ctx->coll_fn(ctx->coll_user, buf, count, op, ctx->stream);
  if (st != 0)
    return fail(ctx, DB200_ERR_COLLECTIVE, "collective all-reduce of " + std::to_string(count) +
                                               " values failed on rank " + std::to_string(ctx->coll_rank) +
                                               " (status " + std::to_string(st) + ")");
  return DB200_OK;
}

}  // namespace db200

using namespace db200;

extern "C" {

int db200_create(db200_context** out, int device, void* stream) {
  if (!out) return DB200_ERR_INVALID;
  *out = nullptr;
  auto* ctx = new db200_context();
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    delete ctx;
    return DB200_ERR_CUDA;
  }
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) {
    delete ctx;
    return DB200_ERR_CUDA;
  }
  if (prop.major != 10) {
    std::fprintf(stderr, "darray_b200: device %d is sm_%d%d; this library is built for sm_100a only\n", device,
                 prop.major, prop.minor);
    delete ctx;
    return DB200_ERR_UNSUPPORTED;
  }
  ctx->num_sms = prop.multiProcessorCount;
  if (stream == DB200_OWN_STREAM) {
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete ctx;
      return DB200_ERR_CUDA;
    }
    ctx->own_stream = true;
  } else {
    ctx->stream = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
  }
  // [0] the status word, [1] the arrival counter of the blocked Cholesky's diagonal-block kernel, [2..3] spare
  if (cudaMalloc(&ctx->d_status, 4 * sizeof(int)) != cudaSuccess ||
      cudaMemsetAsync(ctx->d_status, 0, 4 * sizeof(int), ctx->stream) != cudaSuccess ||
      cudaMallocHost(&ctx->h_pinned, 4096) != cudaSuccess) {
    db200_destroy(ctx);
    return DB200_ERR_CUDA;
  }
  db200::potrf_cluster_init(ctx);
  *out = ctx;
  return DB200_OK;
}

int db200_destroy(db200_context* ctx) {
  if (!ctx) return DB200_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (db200_context* w : ctx->workers) db200_destroy(w);
  ctx->workers.clear();
  prof_clear(ctx);
  for (auto& e : ctx->graphs) cudaGraphExecDestroy(e.exec);
  ctx->graphs.clear();
  if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
  if (ctx->ws) cudaFree(ctx->ws);
  if (ctx->io) cudaFree(ctx->io);
  for (void* p : ctx->slot)
    if (p) cudaFree(p);
  if (ctx->tile_table) cudaFree(ctx->tile_table);
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
  if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return DB200_OK;
}

const char* db200_last_error(const db200_context* ctx) { return ctx ? ctx->last_error.c_str() : "no context"; }

void* db200_stream(const db200_context* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int64_t db200_launch_count(const db200_context* ctx) { return ctx ? (int64_t)ctx->launches : 0; }

int db200_profile(db200_context* ctx, int enable) {
  if (!ctx) return DB200_ERR_INVALID;
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  prof_clear(ctx);
  ctx->profiling = enable != 0;
  return DB200_OK;
}

int db200_profile_read(db200_context* ctx, double* total_ms, int64_t* count) {
  if (!ctx || !total_ms || !count) return DB200_ERR_INVALID;
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  double t = 0;
  for (auto& p : ctx->prof_events) {
    float ms = 0;
    DB200_CUDA(ctx, cudaEventElapsedTime(&ms, p.first, p.second));
    t += ms;
  }
  *total_ms = t;
  *count = (int64_t)ctx->prof_events.size();
  prof_clear(ctx);
  return DB200_OK;
}

int db200_synchronize(db200_context* ctx) {
  if (!ctx) return DB200_ERR_INVALID;
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  int st = 0;
  DB200_CUDA(ctx, cudaMemcpy(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st != 0) {
    cudaMemset(ctx->d_status, 0, sizeof(int));
    return fail(ctx, st, "a device-side bounded wait gave up (kernel pipeline stalled)");
  }
  return DB200_OK;
}

static int check_points(db200_context* ctx, int m, int d, const float* X, int ldx, int layout) {
  if (!X) return fail(ctx, DB200_ERR_INVALID, "null point matrix");
  if (layout == DB200_POINT_MAJOR) {
    if (ldx < d) return fail(ctx, DB200_ERR_INVALID, "point-major ldx < d");
  } else if (layout == DB200_FEATURE_MAJOR) {
    if (ldx < m) return fail(ctx, DB200_ERR_INVALID, "feature-major ldx < m");
  } else {
    return fail(ctx, DB200_ERR_INVALID, "unknown point layout");
  }
  return DB200_OK;
}

// Packs Xi (and Xj unless it is the same matrix) into the workspace.
static int pack_pair(db200_context* ctx, int m, int n, int d, const float* Xi, int ldxi, const float* Xj, int ldxj,
                     int layout, size_t extra_bytes, PackedPoints& pi, PackedPoints& pj, Carve& carve) {
  const int dp = feature_pad(d);
  const int mpad = point_pad(m), npad = point_pad(n);
  const bool same = (Xi == Xj && ldxi == ldxj && m == n);
  size_t bytes = 4096 + (size_t)mpad * (2 * dp * 2 + 8) + extra_bytes + 4 * 256;
  if (!same) bytes += (size_t)npad * (2 * dp * 2 + 8);
  void* ws = workspace(ctx, bytes);
  if (!ws) return DB200_ERR_NOMEM;
  carve = Carve{static_cast<char*>(ws)};
  void* xpi = carve.take<uint16_t>((size_t)mpad * 2 * dp);
  float* ni = carve.take<float>(packed_norm_floats(mpad));
  int st = pack_points(ctx, Xi, ldxi, layout, m, d, dp, mpad, xpi, ni);
  if (st) return st;
  pi.xp = xpi;
  pi.norms = ni;
  pi.n = m;
  pi.npad = mpad;
  pi.dp = dp;
  if (same) {
    pj = pi;
  } else {
    void* xpj = carve.take<uint16_t>((size_t)npad * 2 * dp);
    float* nj = carve.take<float>(packed_norm_floats(npad));
    st = pack_points(ctx, Xj, ldxj, layout, n, d, dp, npad, xpj, nj);
    if (st) return st;
    pj.xp = xpj;
    pj.norms = nj;
    pj.n = n;
    pj.npad = npad;
    pj.dp = dp;
  }
  return DB200_OK;
}

int db200_rbf_sketch_ex(db200_context* ctx, int m, int n, int d, int l, const float* Xi, int ldxi, const float* Xj,
                        int ldxj, int x_layout, const float* yi, const float* yj, const float* Omega, int ldo,
                        float* Y, int ldy, float gamma, int product) {
  if (!ctx) return DB200_ERR_INVALID;
  if (m < 0 || n < 0 || d < 1 || l < 0) return fail(ctx, DB200_ERR_INVALID, "rbf_sketch: negative size");
  if (product < DB200_SKETCH_SINGLE || product > DB200_SKETCH_COMPENSATED_PROMOTED_COARSE)
    return fail(ctx, DB200_ERR_INVALID, "rbf_sketch: unknown sketch product");
  if (m == 0 || l == 0) return DB200_OK;
  if (d > 128) return fail(ctx, DB200_ERR_UNSUPPORTED, "rbf_sketch: d > 128 not supported");
  if (!Y || ldy < m) return fail(ctx, DB200_ERR_INVALID, "rbf_sketch: bad Y / ldy");
  if (n == 0) {
    for (int c = 0; c < l; ++c) DB200_CUDA(ctx, cudaMemsetAsync(Y + (size_t)c * ldy, 0, sizeof(float) * m, ctx->stream));
    return DB200_OK;
  }
  if (!Omega || ldo < n) return fail(ctx, DB200_ERR_INVALID, "rbf_sketch: bad Omega / ldo");
  int st = check_points(ctx, m, d, Xi, ldxi, x_layout);
  if (!st) st = check_points(ctx, n, d, Xj, ldxj, x_layout);
  if (st) return st;
  const bool promoted = product >= DB200_SKETCH_COMPENSATED_PROMOTED;
  SketchPlan plan = plan_sketch(l, promoted ? 2 : product);
  // accumulation chunks of two j tiles (256 points; the truncation loss of the tensor cores' fp32 accumulation
  // stays at ~48 steps x 2^-25 of a value) or, coarse, of eight (1024 points, ~192 steps)
  if (promoted) plan.promote = (product == DB200_SKETCH_COMPENSATED_PROMOTED) ? 2 : 8;
  const int npad = point_pad(n);
  const size_t op_halves = packed_sketch_halves(plan, npad);
  PackedPoints pi, pj;
  Carve carve{nullptr};
  st = pack_pair(ctx, m, n, d, Xi, ldxi, Xj, ldxj, x_layout, op_halves * 2 + 256, pi, pj, carve);
  if (st) return st;
  void* op = carve.take<uint16_t>(op_halves);
  st = pack_sketch(ctx, Omega, ldo, yj, n, l, npad, plan.lrows, op, plan.comp);
  if (st) return st;
  return launch_rbf_sketch_exact(ctx, pi, pj, yi, op, plan, l, gamma, Y, ldy);
}

int db200_rbf_sketch(db200_context* ctx, int m, int n, int d, int l, const float* Xi, int ldxi, const float* Xj,
                     int ldxj, int x_layout, const float* yi, const float* yj, const float* Omega, int ldo, float* Y,
                     int ldy, float gamma) {
  return db200_rbf_sketch_ex(ctx, m, n, d, l, Xi, ldxi, Xj, ldxj, x_layout, yi, yj, Omega, ldo, Y, ldy, gamma,
                             DB200_SKETCH_SINGLE);
}

int db200_rbf_block(db200_context* ctx, int m, int n, int d, const float* Xi, int ldxi, const float* Xj, int ldxj,
                    int x_layout, const float* yi, const float* yj, float* K, int ldk, float gamma) {
  if (!ctx) return DB200_ERR_INVALID;
  if (m < 0 || n < 0 || d < 1) return fail(ctx, DB200_ERR_INVALID, "rbf_block: negative size");
  if (m == 0 || n == 0) return DB200_OK;
  if (d > 128) return fail(ctx, DB200_ERR_UNSUPPORTED, "rbf_block: d > 128 not supported");
  if (!K || ldk < m) return fail(ctx, DB200_ERR_INVALID, "rbf_block: bad K / ldk");
  int st = check_points(ctx, m, d, Xi, ldxi, x_layout);
  if (!st) st = check_points(ctx, n, d, Xj, ldxj, x_layout);
  if (st) return st;
  PackedPoints pi, pj;
  Carve carve{nullptr};
  st = pack_pair(ctx, m, n, d, Xi, ldxi, Xj, ldxj, x_layout, 0, pi, pj, carve);
  if (st) return st;
  SketchPlan plan;
  return launch_rbf_tiles(ctx, RBF_MODE_KBLOCK, pi, pj, yi, yj, nullptr, plan, 0, gamma, K, ldk);
}

int db200_lra_host(db200_context* ctx, int n, int d, int k, const float* X, int ldx, const float* Y,
                   const float* O, int ldo, float* A, int lda, float gamma) {
  if (!ctx) return DB200_ERR_INVALID;
  if (n < 0 || d < 1 || k < 0 || !X || !Y || !O || !A || ldx < d || ldo < n || lda < n)
    return fail(ctx, DB200_ERR_INVALID, "lra_host: bad arguments");
  if (n == 0 || k == 0) return DB200_OK;
  // A result in page-locked host memory that the device can address is written by the kernel itself: its
  // stores drain over the host link while the kernel runs, instead of a copy after it.  Pageable memory takes the
  // staged copy.
  float* direct = nullptr;
  {
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, A) == cudaSuccess && pa.type == cudaMemoryTypeHost && pa.devicePointer)
      direct = static_cast<float*>(pa.devicePointer);
    cudaGetLastError();  // an unregistered pointer may leave an error behind on older drivers
  }
  const size_t bx = align_up(sizeof(float) * (size_t)n * d, 256), by = align_up(sizeof(float) * (size_t)n, 256),
               bo = align_up(sizeof(float) * (size_t)n * k, 256);
  char* io = static_cast<char*>(io_buffer(ctx, bx + by + (direct ? 1 : 2) * bo));
  if (!io) return DB200_ERR_NOMEM;
  float* dX = reinterpret_cast<float*>(io);
  float* dY = reinterpret_cast<float*>(io + bx);
  float* dO = reinterpret_cast<float*>(io + bx + by);
  float* dA = direct ? direct : reinterpret_cast<float*>(io + bx + by + bo);
  const int ldA = direct ? lda : n;
  DB200_CUDA(ctx, cudaMemcpy2DAsync(dX, sizeof(float) * d, X, sizeof(float) * ldx, sizeof(float) * d, n,
                                    cudaMemcpyHostToDevice, ctx->stream));
  DB200_CUDA(ctx, cudaMemcpyAsync(dY, Y, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
  DB200_CUDA(ctx, cudaMemcpy2DAsync(dO, sizeof(float) * n, O, sizeof(float) * ldo, sizeof(float) * n, k,
                                    cudaMemcpyHostToDevice, ctx->stream));
  int st = db200_rbf_sketch(ctx, n, n, d, k, dX, d, dX, d, DB200_POINT_MAJOR, dY, dY, dO, n, dA, ldA, gamma);
  if (st) return st;
  if (!direct)
    DB200_CUDA(ctx, cudaMemcpy2DAsync(A, sizeof(float) * lda, dA, sizeof(float) * n, sizeof(float) * n, k,
                                      cudaMemcpyDeviceToHost, ctx->stream));
  return db200_synchronize(ctx);
}

int db200_set_collective(db200_context* ctx, const db200_collective* c) {
  if (!ctx) return DB200_ERR_INVALID;
  if (!c || c->world <= 1) {
    ctx->coll_world = 1;
    ctx->coll_rank = 0;
    ctx->coll_fn = nullptr;
    ctx->coll_user = nullptr;
    return DB200_OK;
  }
  if (c->rank < 0 || c->rank >= c->world || !c->allreduce)
    return fail(ctx, DB200_ERR_INVALID, "set_collective: rank outside [0, world) or no all-reduce");
  ctx->coll_world = c->world;
  ctx->coll_rank = c->rank;
  ctx->coll_fn = c->allreduce;
  ctx->coll_user = c->user;
  return DB200_OK;
}

int db200_row_shard(int n, int world, int rank, int* start, int* count) {
  if (n < 0 || world < 1 || rank < 0 || rank >= world || !start || !count) return DB200_ERR_INVALID;
  const int base = n / world, extra = n % world;
  *count = base + (rank < extra ? 1 : 0);
  *start = rank * base + (rank < extra ? rank : extra);
  return DB200_OK;
}

}  // extern "C"
