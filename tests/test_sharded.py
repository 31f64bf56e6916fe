"""Host side of the row-sharded path on CPU: the row partition (db200_row_shard, through the C ABI), the all-reduce
callbacks the library calls (darray_optimizer_b200.sharded) on host buffers -- in-process loopback ranks and
torch.distributed over gloo at world size 2 -- and the exchange patterns the sharded solve builds on them: the Gram
of row blocks summed over ranks, Q gathered as a sum of zero-filled row blocks, and the global sums, maxima and
minima of the barrier.  The device side is tests/test_sharded_gpu.py."""
import ctypes
import multiprocessing as mp
import os
import socket
import threading

import numpy as np
import pytest

from darray_optimizer_b200 import sharded


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p).value


@pytest.mark.parametrize("n", [0, 1, 7, 100, 4096, 131072])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_row_shard_partition(n, world):
    blocks = [sharded.row_shard(n, world, k) for k in range(world)]
    pos = 0
    for s, c in blocks:
        assert s == pos and c >= 0
        pos += c
    assert pos == n
    counts = [c for _, c in blocks]
    assert max(counts) - min(counts) <= 1


def test_row_shard_rejects_bad_arguments():
    from darray_optimizer_b200._lib import DB200Error
    for args in [(-1, 2, 0), (10, 0, 0), (10, 2, 2), (10, 2, -1)]:
        with pytest.raises(DB200Error):
            sharded.row_shard(*args)


def _gather_by_sum(call, Q_rows, n, l, start):
    """All rows of Q from this rank's block: its rows at their offset in a zero matrix, summed over the ranks (the
    gather of the power and final passes)."""
    full = np.zeros((l, n))  # column major n x l: column c is full[c]
    full[:, start:start + Q_rows.shape[0]] = Q_rows.T
    flat = np.ascontiguousarray(full).reshape(-1)
    call(flat, sharded.SUM)
    return flat.reshape(l, n).T


def _patterns(world, rank, call, seed=5):
    """The sharded solve's exchanges on host data; returns what every rank must agree on."""
    n, l = 101, 6
    g = np.random.default_rng(seed)
    Y = g.standard_normal((n, l))
    s, c = sharded.row_shard(n, world, rank)
    out = {}
    # Gram of CholeskyQR2 / the Nystrom core: sum of the ranks' block Grams
    G = np.ascontiguousarray(Y[s:s + c].T @ Y[s:s + c]).reshape(-1)
    call(G, sharded.SUM)
    out["gram"] = G.reshape(l, l)
    out["gram_ref"] = Y.T @ Y
    out["gather"] = _gather_by_sum(call, Y[s:s + c], n, l, s)
    out["gather_ref"] = Y
    # barrier scalars: [sum a, sum logs] summed, max D, min D
    a = np.abs(Y[:, 0]) + 0.1
    v = np.array([a[s:s + c].sum(), np.log(a[s:s + c]).sum()])
    call(v, sharded.SUM)
    mx = np.array([a[s:s + c].max() if c else 0.0])
    call(mx, sharded.MAX)
    mn = np.array([a[s:s + c].min() if c else np.finfo(np.float64).max])
    call(mn, sharded.MIN)
    out["scalars"] = np.concatenate([v, mx, mn])
    out["scalars_ref"] = np.array([a.sum(), np.log(a).sum(), a.max(), a.min()])
    return out


def _check(out):
    np.testing.assert_allclose(out["gram"], out["gram_ref"], rtol=1e-12, atol=1e-12)
    assert np.array_equal(out["gather"], out["gather_ref"])  # one non-zero term per entry: exact
    np.testing.assert_allclose(out["scalars"], out["scalars_ref"], rtol=1e-12)


def test_loopback_collective_on_host_buffers():
    world = 3
    coll = sharded.LoopbackCollective(world, device="cpu", timeout=30)
    results, errors = [None] * world, []

    def run(k):
        try:
            fn = coll.rank(k).fn

            def call(buf, op):
                assert fn(None, _ptr(buf), buf.size, op, None) == 0

            results[k] = _patterns(world, k, call)
        except BaseException as e:
            errors.append(e)

    ts = [threading.Thread(target=run, args=(k,)) for k in range(world)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=60)
    assert not errors, errors
    for out in results:
        _check(out)
    assert all(coll.rank(k).calls == 5 for k in range(world))


def test_loopback_collective_reports_disagreement():
    """Ranks that call with different counts make every rank's call fail (status != 0), not hang."""
    coll = sharded.LoopbackCollective(2, device="cpu", timeout=30)
    status = [None, None]

    def run(k):
        buf = np.ones(3 + k)
        status[k] = coll.rank(k).fn(None, _ptr(buf), buf.size, sharded.SUM, None)

    ts = [threading.Thread(target=run, args=(k,)) for k in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=60)
    assert status[0] != 0 and status[1] != 0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_worker(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import datetime

    import torch.distributed as dist
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
        coll = sharded.TorchCollective(device="cpu")

        def call(buf, op):
            st = coll.fn(None, _ptr(buf), buf.size, op, None)
            if st != 0:
                raise RuntimeError(f"collective failed: {coll.error!r}")

        out = _patterns(world, rank, call)
        _check(out)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, "ok", coll.calls, coll.values))
    except Exception as e:  # reported, so that the test fails instead of hanging
        q.put((rank, "error", type(e).__name__, str(e)[:300]))


def test_torch_collective_gloo_world_two():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert [r[1] for r in res] == ["ok", "ok"], res
    # the same exchanges on both ranks: 5 calls of 36 + 606 + 2 + 1 + 1 values
    assert res[0][2:] == res[1][2:] == (5, 36 + 606 + 4)
