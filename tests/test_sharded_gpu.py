"""Row-sharded solve on one GPU: `world` ranks as threads of this process (LoopbackCollective), each with its own
context and stream and its own rows of the problem, against the unsharded solve on the same inputs.

The ranks exchange only through the host-side rendezvous of the loopback all-reduce, after each rank's stream has
been synchronised: no kernel waits on another rank.  Checks, on the two-Gaussian workload (n = 4096, d = 32,
l = 138, q = 1, C = 1):
  * FP64 (DB200_FP64): the rows of Z from every rank stacked equal the unsharded factor to 1e-9 (the same
    arithmetic, sums split at the rank boundaries), and the dual objective to 1e-9;
  * mixed (DB200_MIXED): dual objective within 1e-6 of the unsharded solve's and of the oracle's, the gaps
    <= 1e-6 on every rank, and every rank reports the same objective;
  * the barrier alone over row blocks of one fixed factor (world 3, uneven blocks) against db200_svm_barrier on the
    whole factor: objective to 1e-10 and the dual vectors stacked to 1e-7 in FP64 (1e-8 and 1e-5 mixed);
  * a solve with a collective attached refuses the learned-landmark path.
"""
import threading

import numpy as np
import pytest

from darray_optimizer_b200 import datagen, sharded
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dev(a, dtype):
    import torch
    a = np.asarray(a, dtype)
    if a.ndim == 2:
        return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()  # column major
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _run_ranks(world, body):
    """body(ctx, rank) in `world` threads, each with its own context and stream, collective attached."""
    import torch
    from darray_optimizer_b200._lib import Context
    coll = sharded.LoopbackCollective(world, device="cuda", timeout=120)
    results, errors = [None] * world, []

    def run(k):
        try:
            stream = torch.cuda.Stream()
            with torch.cuda.stream(stream):
                ctx = Context(0, stream.cuda_stream)
                coll.attach(ctx, k)
                results[k] = body(ctx, k)
                ctx.set_collective(1, 0)
                ctx.close()
        except BaseException as e:
            errors.append((k, e, coll.rank(k).error))

    ts = [threading.Thread(target=run, args=(k,)) for k in range(world)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=600)
    assert not errors, errors
    return results


@pytest.fixture(scope="module")
def problem():
    w = datagen.two_gaussians(n=4096, d=32, seed=1)
    return w, w.omega()


def _unsharded(gpu_ctx, w, Om, precision):
    import torch
    n, l = w.n, w.l
    dX, dy, dO = _dev(w.X.T, np.float32), _dev(w.y, np.float32), _dev(Om, np.float32)
    dZ = torch.zeros((l, n), dtype=torch.float64, device="cuda")
    da = torch.zeros(n, dtype=torch.float64, device="cuda")
    rep = gpu_ctx.svm_solve(n, w.d, l, w.power_iters, dX.data_ptr(), w.d, dy.data_ptr(), dO.data_ptr(), n, w.gamma,
                            w.C, da.data_ptr(), dZ.data_ptr(), n, params=gpu_ctx.barrier_params(precision=precision))
    return rep, dZ.cpu().numpy().T, da.cpu().numpy()


def _sharded_solve(world, w, Om, precision):
    import torch
    n, l = w.n, w.l

    def body(ctx, k):
        s, c = sharded.row_shard(n, world, k)
        dX, dy, dO = _dev(w.X.T, np.float32), _dev(w.y, np.float32), _dev(Om, np.float32)
        dZ = torch.zeros((l, c), dtype=torch.float64, device="cuda")  # this rank's rows, ldz = c
        da = torch.zeros(c, dtype=torch.float64, device="cuda")
        rep = ctx.svm_solve(n, w.d, l, w.power_iters, dX.data_ptr(), w.d, dy.data_ptr(), dO.data_ptr(), n, w.gamma,
                            w.C, da.data_ptr(), dZ.data_ptr(), c, params=ctx.barrier_params(precision=precision))
        torch.cuda.current_stream().synchronize()
        return rep, dZ.cpu().numpy().T, da.cpu().numpy()

    res = _run_ranks(world, body)
    return [r[0] for r in res], np.vstack([r[1] for r in res]), np.concatenate([r[2] for r in res])


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_solve_fp64_matches_unsharded(gpu_ctx, problem, world):
    w, Om = problem
    rep1, Z1, a1 = _unsharded(gpu_ctx, w, Om, precision=1)
    reps, Z, a = _sharded_solve(world, w, Om, precision=1)
    assert np.linalg.norm(Z - Z1) <= 1e-9 * np.linalg.norm(Z1)
    for rep in reps:
        assert rep.status == 0
        assert rep.f == reps[0].f  # every rank reports the same (all-reduced) objective
        assert abs(rep.f - rep1.f) <= 1e-9 * abs(rep1.f)
        assert rep.gap_barrier < 1e-6 and rep.gap_primal_dual < 1e-6
    assert np.all(a > 0) and np.all(a < w.C)


def test_sharded_solve_mixed_matches_unsharded_and_oracle(gpu_ctx, problem):
    w, Om = problem
    rep1, _, _ = _unsharded(gpu_ctx, w, Om, precision=0)
    reps, Z, a = _sharded_solve(2, w, Om, precision=0)
    lr = O.low_rank_factor(w.X, w.y, Om, w.gamma, w.power_iters)
    ref = O.svm_barrier(lr.Z, w.y, w.C)
    for rep in reps:
        assert rep.status == 0 and rep.f == reps[0].f
        assert rep.gap_barrier < 1e-6 and rep.gap_primal_dual < 1e-6
    f = reps[0].f
    print(f"sharded mixed: |f - f_unsharded|/|f| = {abs(f - rep1.f) / abs(rep1.f):.3e}, "
          f"|f - f_oracle|/|f_oracle| = {abs(f - ref.f) / abs(ref.f):.3e}")
    assert abs(f - rep1.f) <= 1e-6 * abs(rep1.f)
    assert abs(f - ref.f) <= 1e-6 * abs(ref.f)


@pytest.mark.parametrize("precision", [0, 1])
def test_sharded_barrier_matches_whole_factor(gpu_ctx, precision):
    import torch
    w = datagen.two_gaussians(n=2048, d=16, seed=4)
    w.rank, w.oversample = 48, 8
    lr = O.low_rank_factor(w.X, w.y, w.omega(), w.gamma, w.power_iters)
    n, r = lr.Z.shape
    dZ, dy = _dev(lr.Z, np.float64), _dev(w.y, np.float32)
    da = torch.zeros(n, dtype=torch.float64, device="cuda")
    rep1 = gpu_ctx.svm_barrier(n, r, dZ.data_ptr(), n, dy.data_ptr(), w.C, da.data_ptr(),
                               params=gpu_ctx.barrier_params(precision=precision))
    a1 = da.cpu().numpy()
    world = 3  # 683 + 683 + 682 rows

    def body(ctx, k):
        s, c = sharded.row_shard(n, world, k)
        Zk = _dev(lr.Z[s:s + c], np.float64)
        yk = _dev(w.y[s:s + c], np.float32)
        ak = torch.zeros(c, dtype=torch.float64, device="cuda")
        rep = ctx.svm_barrier(c, r, Zk.data_ptr(), c, yk.data_ptr(), w.C, ak.data_ptr(),
                              params=ctx.barrier_params(precision=precision))
        torch.cuda.current_stream().synchronize()
        return rep, ak.cpu().numpy()

    res = _run_ranks(world, body)
    a = np.concatenate([x[1] for x in res])
    # FP64: the same steps, sums split at the rank boundaries; mixed: the int8 capacity matrix of each rank's rows,
    # refined against the exact operator to 1e-10 at every step
    ftol, atol = (1e-10, 1e-7) if precision == 1 else (1e-8, 1e-5)
    for rep, _ in res:
        assert rep.status == 0 and rep.f == res[0][0].f and rep.newton == res[0][0].newton
        assert abs(rep.f - rep1.f) <= ftol * abs(rep1.f)
        assert rep.gap_primal_dual < 1e-6
    assert np.linalg.norm(a - a1) <= atol * np.linalg.norm(a1)


def test_landmark_solve_refuses_while_sharded(gpu_ctx):
    # the refusal comes before any argument is read
    statuses = _run_ranks(2, lambda ctx, k: ctx.lib.db200_svm_solve_landmarks(
        ctx.h, 100, 4, 10, None, 4, None, 0.5, 1.0, None, 0, 16, 16, 0.1, None, 100, 26, 1, None, None, None, 100,
        None, None))
    assert statuses == [-8, -8]  # DB200_ERR_UNSUPPORTED
