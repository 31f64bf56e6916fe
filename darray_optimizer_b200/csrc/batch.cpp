// Batched instances: many independent sketch problems / SVM solves in single persistent launches of the tile
// engine, with the repeated kernel pass captured once in a CUDA graph and the per-instance barriers on worker
// threads.  No counterpart in the reference, which runs one problem per process (tests/testsvm.cpp:34-329).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

#include "internal.h"
#include "la64.h"

namespace db200 {
namespace {

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s;
  explicit Timer(cudaStream_t st) : s(st) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
  }
  double stop() {
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

// Tile plan of one problem: explicit (validated by prepare_rbf_tiles) or the default heuristic.
SketchPlan job_plan(int l, int n_panels, int panel, int g_bufs) {
  if (n_panels <= 0) return plan_sketch(l);
  SketchPlan p;
  p.n_panels = n_panels;
  p.panel = panel;
  p.g_bufs = g_bufs;
  p.lrows = n_panels * panel;
  return p;
}

// Device layout of one batched problem's packed operands.
struct Packed {
  PackedPoints pi, pj;
  void* op = nullptr;
  SketchPlan plan;
  int npad_i = 0, npad_j = 0;
};

size_t packed_bytes(int m, int n, int d, bool same, const SketchPlan& plan) {
  const int dp = feature_pad(d), mpad = point_pad(m), npad = point_pad(n);
  size_t b = align_up((size_t)mpad * 2 * dp * 2, 256) + align_up(packed_norm_floats(mpad) * 4, 256);
  if (!same) b += align_up((size_t)npad * 2 * dp * 2, 256) + align_up(packed_norm_floats(npad) * 4, 256);
  b += align_up(packed_sketch_halves(plan, npad) * 2, 256);
  return b;
}

// The plan of a compensated sketch (comp = 2) with promoted accumulation: the explicit plan when it leaves tensor
// memory for P_lo and takes one instruction per panel, else the default compensated plan.
SketchPlan comp_plan(const SketchPlan& p, int l) {
  SketchPlan c = p;
  c.comp = 2;
  if (!(c.panel <= 256 && c.panel + 128 + 128 * c.g_bufs <= 512)) c = plan_sketch(l, 2);
  c.promote = 8;  // range-finder passes: accumulation promoted every eight j tiles, as in db200_lowrank
  return c;
}

int pack_problem(db200_context* ctx, int m, int n, int d, const float* Xi, int ldxi, const float* Xj, int ldxj,
                 const SketchPlan& plan, Carve& cv, Packed* P) {
  const int dp = feature_pad(d), mpad = point_pad(m), npad = point_pad(n);
  const bool same = (Xi == Xj && ldxi == ldxj && m == n);
  void* xpi = cv.take<uint16_t>((size_t)mpad * 2 * dp);
  float* ni = cv.take<float>(packed_norm_floats(mpad));
  int st = pack_points(ctx, Xi, ldxi, DB200_POINT_MAJOR, m, d, dp, mpad, xpi, ni);
  if (st) return st;
  P->pi.xp = xpi;
  P->pi.norms = ni;
  P->pi.n = m;
  P->pi.npad = mpad;
  P->pi.dp = dp;
  if (same) {
    P->pj = P->pi;
  } else {
    void* xpj = cv.take<uint16_t>((size_t)npad * 2 * dp);
    float* nj = cv.take<float>(packed_norm_floats(npad));
    if ((st = pack_points(ctx, Xj, ldxj, DB200_POINT_MAJOR, n, d, dp, npad, xpj, nj))) return st;
    P->pj.xp = xpj;
    P->pj.norms = nj;
    P->pj.n = n;
    P->pj.npad = npad;
    P->pj.dp = dp;
  }
  P->op = cv.take<uint16_t>(packed_sketch_halves(plan, npad));
  P->plan = plan;
  P->npad_i = mpad;
  P->npad_j = npad;
  return DB200_OK;
}

}  // namespace
}  // namespace db200

using namespace db200;

extern "C" {

int db200_rbf_sketch_batched(db200_context* ctx, int count, const db200_sketch_job* jobs) {
  if (!ctx) return DB200_ERR_INVALID;
  if (count < 0 || (count > 0 && !jobs)) return fail(ctx, DB200_ERR_INVALID, "rbf_sketch_batched: bad arguments");
  if (count == 0) return DB200_OK;
  size_t bytes = 4096;
  std::vector<SketchPlan> plans((size_t)count);
  for (int b = 0; b < count; ++b) {
    const db200_sketch_job& J = jobs[b];
    if (J.m < 1 || J.n < 1 || J.d < 1 || J.d > 128 || J.l < 1 || !J.Xi || !J.Xj || J.ldxi < J.d || J.ldxj < J.d ||
        !J.Omega || J.ldo < J.n || !J.Y || J.ldy < J.m)
      return fail(ctx, DB200_ERR_INVALID, "rbf_sketch_batched: bad job " + std::to_string(b));
    plans[(size_t)b] = job_plan(J.l, J.n_panels, J.panel, J.g_bufs);
    bytes += packed_bytes(J.m, J.n, J.d, J.Xi == J.Xj && J.ldxi == J.ldxj && J.m == J.n, plans[(size_t)b]);
  }
  void* ws = workspace(ctx, bytes);
  if (!ws) return DB200_ERR_NOMEM;
  Carve cv{static_cast<char*>(ws)};
  std::vector<TileJob> tj((size_t)count);
  for (int b = 0; b < count; ++b) {
    const db200_sketch_job& J = jobs[b];
    Packed P;
    int st = pack_problem(ctx, J.m, J.n, J.d, J.Xi, J.ldxi, J.Xj, J.ldxj, plans[(size_t)b], cv, &P);
    if (!st) st = pack_sketch(ctx, J.Omega, J.ldo, J.yj, J.n, J.l, P.npad_j, P.plan.lrows, P.op);
    if (st) return st;
    TileJob& T = tj[(size_t)b];
    T.pi = P.pi;
    T.pj = P.pj;
    T.yi = J.yi;
    T.yj = nullptr;  // folded into the packed Omega
    T.op = P.op;
    T.plan = P.plan;
    T.l = J.l;
    T.gamma = J.gamma;
    T.out = J.Y;
    T.ldo = J.ldy;
  }
  TilePlan plan;
  int st = prepare_rbf_tiles(ctx, RBF_MODE_SKETCH, tj.data(), count, nullptr, 0, &plan);
  if (st) return st;
  return launch_rbf_plan(ctx, plan);
}

int db200_svm_solve_batched(db200_context* ctx, int count, const db200_svm_instance* inst, int q,
                            const db200_barrier_params* params, int use_graph, int workers,
                            db200_svm_report* reports, db200_batch_report* brep) {
  if (!ctx) return DB200_ERR_INVALID;
  if (count < 1 || !inst || q < 0 || q > 8) return fail(ctx, DB200_ERR_INVALID, "svm_solve_batched: bad arguments");
  for (int b = 0; b < count; ++b) {
    const db200_svm_instance& I = inst[b];
    if (I.n < 2 || I.d < 1 || I.d > 128 || I.l < 1 || I.l > I.n || !I.X || I.ldx < I.d || !I.y || !(I.C > 0) ||
        !I.Omega || I.ldo < I.n || !I.Z || I.ldz < I.n || !I.a)
      return fail(ctx, DB200_ERR_INVALID, "svm_solve_batched: bad instance " + std::to_string(b));
  }
  db200_batch_report R;
  std::memset(&R, 0, sizeof(R));
  db200_barrier_params P;
  if (params) P = *params;
  else db200_barrier_defaults(&P);
  const auto wall0 = std::chrono::steady_clock::now();
  auto wall_ms = [](std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  };

  if (workers < 1) workers = 1;
  if (workers > count) workers = count;
  R.workers = workers;

  // ---- device buffers: packed points and test matrices (workspace), per-instance pass outputs (pipeline slot)
  std::vector<SketchPlan> plans((size_t)count);
  size_t wbytes = 4096, pbytes = 4096 + (size_t)workers * 256;  // + the final pass's instance table, below
  int njobs = 0;  // tile-engine instances: default multi-panel plans split into exact-width panels
  for (int b = 0; b < count; ++b) {
    const db200_svm_instance& I = inst[b];
    plans[(size_t)b] = job_plan(I.l, I.n_panels, I.panel, I.g_bufs);
    // kernel passes with the compensated sketch product unless the fast mixed form is asked for
    if (P.precision != DB200_MIXED_FAST) plans[(size_t)b] = comp_plan(plans[(size_t)b], I.l);
    wbytes += packed_bytes(I.n, I.n, I.d, true, plans[(size_t)b]);
    njobs += (I.n_panels <= 0) ? plans[(size_t)b].n_panels : 1;
    const size_t nl = (size_t)I.n * I.l, ll = (size_t)I.l * I.l;
    pbytes += 2 * align_up(nl * 4, 256) + align_up(nl * 8, 256) + 2 * align_up(ll * 8, 256);
  }
  wbytes += align_up(tile_table_bytes(njobs), 256);
  void* ws = workspace(ctx, wbytes);
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_PIPE, pbytes + 4096));
  if (!ws || !base) return DB200_ERR_NOMEM;
  Carve cw{static_cast<char*>(ws)};
  Carve cp{base};
  // status pair and scalar of the Nystrom core, one set per worker
  std::vector<int*> wpair((size_t)workers);
  std::vector<double*> wscalar((size_t)workers);
  for (int k = 0; k < workers; ++k) {
    wpair[(size_t)k] = cp.take<int>(4);
    wscalar[(size_t)k] = cp.take<double>(4);
  }
  std::vector<Packed> pk((size_t)count);
  std::vector<float*> Y32((size_t)count), Qf((size_t)count);
  std::vector<double*> Q((size_t)count), Cm((size_t)count), Rm((size_t)count);
  int st = DB200_OK;
  {
    Timer t(ctx->stream);
    for (int b = 0; b < count && !st; ++b) {
      const db200_svm_instance& I = inst[b];
      st = pack_problem(ctx, I.n, I.n, I.d, I.X, I.ldx, I.X, I.ldx, plans[(size_t)b], cw, &pk[(size_t)b]);
      const size_t nl = (size_t)I.n * I.l, ll = (size_t)I.l * I.l;
      Y32[(size_t)b] = cp.take<float>(nl);
      Qf[(size_t)b] = cp.take<float>(nl);
      Q[(size_t)b] = cp.take<double>(nl);
      Cm[(size_t)b] = cp.take<double>(ll);
      Rm[(size_t)b] = cp.take<double>(ll);
    }
    if (st) return st;
    R.ms_pack = t.stop();
  }
  // Tile-engine instances.  A default plan of several panels is split into exact-width panels, as the
  // single-problem path splits it, so each instance's passes are the single solve's to the bit; an explicit
  // (autotuned) plan is kept as one instance of equal panels.
  std::vector<TileJob> tj;
  tj.reserve((size_t)njobs);
  for (int b = 0; b < count; ++b) {
    TileJob T;
    T.pi = pk[(size_t)b].pi;
    T.pj = pk[(size_t)b].pj;
    T.yi = inst[b].y;
    T.op = pk[(size_t)b].op;
    T.plan = pk[(size_t)b].plan;
    T.om_lo = T.plan.lrows;
    T.l = inst[b].l;
    T.gamma = inst[b].gamma;
    T.out = Y32[(size_t)b];
    T.ldo = inst[b].n;
    if (inst[b].n_panels <= 0) exact_panel_jobs(T, tj);
    else tj.push_back(T);
  }
  const int nj = (int)tj.size();
  TilePlan tplan, tplan_final;
  if ((st = prepare_rbf_tiles(ctx, RBF_MODE_SKETCH, tj.data(), nj, nullptr, 0, &tplan))) return st;
  // the final pass (Y = K Q, contracted into the Nystrom core, whose scale the accumulation's truncation would
  // shrink) promotes every two j tiles, as db200_lowrank's final pass does; its instance table is in the workspace
  for (TileJob& T : tj)
    if (T.plan.comp == 2) T.plan.promote = 2;
  {
    void* table_final = cw.take<char>(tile_table_bytes(nj));
    if ((st = prepare_rbf_tiles(ctx, RBF_MODE_SKETCH, tj.data(), nj, table_final, tile_table_bytes(nj),
                                &tplan_final)))
      return st;
  }

  // ---- one kernel pass over every instance: pack each test matrix (Omega, or Q from the previous pass), then one
  // persistent launch.  After the first Q pass the sequence is captured once and replayed.
  auto enqueue_pass = [&](bool from_omega, const TilePlan& tp) -> int {
    for (int b = 0; b < count; ++b) {
      const db200_svm_instance& I = inst[b];
      const float* src = from_omega ? I.Omega : Qf[(size_t)b];
      const int lds = from_omega ? I.ldo : I.n;
      int s2 = pack_sketch(ctx, src, lds, I.y, I.n, I.l, pk[(size_t)b].npad_j, pk[(size_t)b].plan.lrows,
                           pk[(size_t)b].op, pk[(size_t)b].plan.comp);
      if (s2) return s2;
    }
    return launch_rbf_plan(ctx, tp);
  };
  cudaStream_t cs = nullptr;
  cudaGraphExec_t graphs[2] = {nullptr, nullptr};  // the range-finder Q pass and the final pass
  cudaEvent_t ev = nullptr;
  auto cleanup = [&]() {
    for (cudaGraphExec_t& g : graphs)
      if (g) cudaGraphExecDestroy(g);
    if (cs) cudaStreamDestroy(cs);
    if (ev) cudaEventDestroy(ev);
  };
  auto q_pass = [&](bool final_pass) -> int {
    const TilePlan& tp = final_pass ? tplan_final : tplan;
    if (!use_graph) return enqueue_pass(false, tp);
    cudaGraphExec_t& gx = graphs[final_pass ? 1 : 0];
    if (!gx) {
      // capture on a private stream (the context's stream may be the legacy default stream)
      if (!cs && (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess ||
                  cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess))
        return fail(ctx, DB200_ERR_CUDA, "svm_solve_batched: stream for graph capture");
      cudaStream_t keep = ctx->stream;
      const bool prof = ctx->profiling;
      const long long launches = ctx->launches;  // captured launches run (and are counted) when replayed
      ctx->stream = cs;
      ctx->profiling = false;
      cudaGraph_t g = nullptr;
      int s2 = DB200_OK;
      if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        s2 = fail(ctx, DB200_ERR_CUDA, "svm_solve_batched: begin capture");
      } else {
        s2 = enqueue_pass(false, tp);
        const cudaError_t e = cudaStreamEndCapture(cs, &g);
        if (!s2 && e != cudaSuccess) s2 = cuda_fail(ctx, e, "cudaStreamEndCapture");
      }
      ctx->stream = keep;
      ctx->profiling = prof;
      ctx->launches = launches;
      if (!s2 && cudaGraphInstantiate(&gx, g, 0) != cudaSuccess)
        s2 = fail(ctx, DB200_ERR_CUDA, "svm_solve_batched: graph instantiate");
      if (g) cudaGraphDestroy(g);
      if (s2) return s2;
    }
    // order the replay after the work already queued on the context's stream, and the rest after it
    DB200_CUDA(ctx, cudaEventRecord(ev, ctx->stream));
    DB200_CUDA(ctx, cudaStreamWaitEvent(cs, ev, 0));
    DB200_CUDA(ctx, cudaGraphLaunch(gx, cs));
    DB200_CUDA(ctx, cudaEventRecord(ev, cs));
    DB200_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ev, 0));
    count_launch(ctx, count + 1);
    R.graph_replays += 1;
    return DB200_OK;
  };
  // ---- worker contexts (own stream and buffers each), kept across calls so their buffers stay grown
  if (workers > 1) {
    while ((int)ctx->workers.size() < workers) {
      db200_context* w = nullptr;
      const int cst = db200_create(&w, ctx->device, DB200_OWN_STREAM);
      if (cst) {
        cleanup();
        return fail(ctx, cst, "svm_solve_batched: worker context");
      }
      ctx->workers.push_back(w);
    }
  }
  // Every worker's CholeskyQR2 and barrier buffers sized for the largest instance now: grown on demand, they would
  // be reallocated whenever a worker met a larger instance than before, and each cudaFree / cudaMalloc stalls the
  // whole device, i.e. every other worker (orthonormalisation 130 ms in one call, 770 ms in another).
  {
    size_t la = 0, bar = 0;
    const bool mixed = (P.precision != DB200_FP64);
    for (int b = 0; b < count; ++b) {
      la = std::max(la, cholqr2_slot_bytes(inst[b].n, inst[b].l));
      bar = std::max(bar, barrier_slot_bytes(inst[b].n, inst[b].l, mixed));
    }
    for (int k = 0; k < workers; ++k) {
      db200_context* w = (workers == 1) ? ctx : ctx->workers[(size_t)k];
      if (!slot_buffer(w, SLOT_LA, la) || !slot_buffer(w, SLOT_BAR, bar)) {
        cleanup();
        return fail(ctx, DB200_ERR_NOMEM, "svm_solve_batched: worker buffers");
      }
    }
  }
  // largest instances first (LPT): the per-instance work grows with n l^2
  std::vector<int> order((size_t)count);
  for (int b = 0; b < count; ++b) order[(size_t)b] = b;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return (double)inst[x].n * inst[x].l * inst[x].l > (double)inst[y].n * inst[y].l * inst[y].l;
  });
  // Per-instance work fn(worker context, worker index, instance) on the worker pool, ordered after everything
  // queued on the context's stream, with the context's stream ordered after all of it.  The steps of one instance
  // (a few dozen small, latency-bound launches and host readbacks) overlap with other instances' this way.
  auto parallel = [&](auto&& fn) -> int {
    if (workers == 1) {
      for (int k = 0; k < count; ++k) {
        const int s2 = fn(ctx, 0, order[(size_t)k]);
        if (s2) return s2;
      }
      return DB200_OK;
    }
    std::vector<cudaEvent_t> done((size_t)workers, nullptr);
    cudaEvent_t ready = nullptr;
    if (cudaEventCreateWithFlags(&ready, cudaEventDisableTiming) != cudaSuccess)
      return fail(ctx, DB200_ERR_CUDA, "svm_solve_batched: event");
    for (auto& e : done) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    cudaEventRecord(ready, ctx->stream);
    std::atomic<int> nxt{0};
    std::vector<int> wst((size_t)workers, DB200_OK);
    std::vector<std::thread> th;
    for (int k = 0; k < workers; ++k)
      th.emplace_back([&, k]() {
        db200_context* w = ctx->workers[(size_t)k];
        if (cudaStreamWaitEvent(w->stream, ready, 0) != cudaSuccess) {
          wst[(size_t)k] = fail(w, DB200_ERR_CUDA, "svm_solve_batched: stream wait");
          return;
        }
        for (int i = nxt.fetch_add(1); i < count && !wst[(size_t)k]; i = nxt.fetch_add(1))
          wst[(size_t)k] = fn(w, k, order[(size_t)i]);
        cudaEventRecord(done[(size_t)k], w->stream);
      });
    for (std::thread& t : th) t.join();
    int s2 = DB200_OK;
    for (int k = 0; k < workers; ++k) {
      cudaStreamWaitEvent(ctx->stream, done[(size_t)k], 0);
      if (!s2 && wst[(size_t)k]) s2 = fail(ctx, wst[(size_t)k], ctx->workers[(size_t)k]->last_error);
    }
    // destroying an event whose record is still pending is deferred by the runtime until it completes
    for (auto& e : done) cudaEventDestroy(e);
    cudaEventDestroy(ready);
    return s2;
  };
  auto orth_all = [&]() -> int {
    Timer t(ctx->stream);
    const int s2 = parallel([&](db200_context* w, int, int b) -> int {
      const db200_svm_instance& I = inst[b];
      int s3 = convert<float, double>(w, Y32[(size_t)b], I.n, Q[(size_t)b], I.n, I.n, I.l);
      if (!s3) s3 = cholqr2_impl(w, I.n, I.l, Q[(size_t)b], I.n, nullptr, 0, false);  // small n: FP64 Grams
      if (!s3) s3 = convert<double, float>(w, Q[(size_t)b], I.n, Qf[(size_t)b], I.n, I.n, I.l);
      return s3;
    });
    if (s2) return s2;
    R.ms_orth += t.stop();
    return DB200_OK;
  };
  {
    Timer t(ctx->stream);
    st = enqueue_pass(true, tplan);
    R.kernel_passes += 1;
    if (!st) R.ms_sketch += t.stop();
  }
  if (!st) st = orth_all();
  for (int it = 0; it < q && !st; ++it) {
    Timer t(ctx->stream);
    st = q_pass(false);
    R.kernel_passes += 1;
    if (!st) R.ms_sketch += t.stop();
    if (!st) st = orth_all();
  }
  if (!st) {  // Y = K Q, the pass the Nystrom core contracts
    Timer t(ctx->stream);
    st = q_pass(true);
    R.kernel_passes += 1;
    if (!st) R.ms_sketch += t.stop();
  }
  if (st) {
    cleanup();
    return st;
  }
  std::vector<double> nus((size_t)count, 0.0);
  {
    Timer t(ctx->stream);
    st = parallel([&](db200_context* w, int k, int b) -> int {
      const db200_svm_instance& I = inst[b];
      return nystrom_core<float>(w, I.n, I.l, Q[(size_t)b], Y32[(size_t)b], Cm[(size_t)b], Rm[(size_t)b],
                                 wpair[(size_t)k], wscalar[(size_t)k], I.Z, I.ldz, &nus[(size_t)b]);
    });
    R.ms_core = t.stop();
  }
  cleanup();
  if (st) return st;
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));

  // ---- barriers: workers pull instances off a shared counter, largest first, each on its own context and stream
  std::vector<db200_svm_report> rep((size_t)count);
  std::vector<int> status((size_t)count, DB200_OK);
  std::atomic<int> next{0};
  auto run = [&](db200_context* w) {
    for (int k = next.fetch_add(1); k < count; k = next.fetch_add(1)) {
      const int b = order[(size_t)k];
      const db200_svm_instance& I = inst[b];
      std::memset(&rep[(size_t)b], 0, sizeof(db200_svm_report));
      status[(size_t)b] = db200_svm_barrier(w, I.n, I.l, I.Z, I.ldz, I.y, I.C, &P, I.a, &rep[(size_t)b]);
      rep[(size_t)b].nu = nus[(size_t)b];
    }
  };
  const auto wall_b = std::chrono::steady_clock::now();
  if (workers == 1) {
    run(ctx);
  } else {
    std::vector<std::thread> th;
    for (int k = 0; k < workers; ++k) th.emplace_back([&, k]() { run(ctx->workers[(size_t)k]); });
    for (std::thread& t : th) t.join();
  }
  R.ms_barrier = wall_ms(wall_b);
  R.ms_total = wall_ms(wall0);
  if (reports)
    for (int b = 0; b < count; ++b) reports[b] = rep[(size_t)b];
  if (brep) *brep = R;
  for (int b = 0; b < count; ++b)
    if (status[(size_t)b] && status[(size_t)b] != DB200_ERR_MAXITER)
      return fail(ctx, status[(size_t)b], "svm_solve_batched: barrier of instance " + std::to_string(b) + " failed");
  for (int b = 0; b < count; ++b)
    if (status[(size_t)b]) return status[(size_t)b];
  return DB200_OK;
}

}  // extern "C"
