"""The N > 1 path of bench.py (independent replicas, one per rank) on CPU with gloo, world size 2: barrier,
max-over-ranks timing and the whole-job aggregate, plus a rank that fails before the collective."""
import multiprocessing as mp
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q, fail_rank):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from darray_optimizer_b200 import replicas
    try:
        r = replicas.init(backend="gloo", timeout_s=10)
        if rank == fail_rank:
            raise RuntimeError("injected failure before the timing collective")
        replicas.barrier(r)
        secs = 1.0 + rank  # rank 1 is the slow one
        tmax = replicas.all_max(r, secs)
        agg = replicas.whole_job_throughput(r, 100.0, secs)
        replicas.barrier(r)
        replicas.finalize(r)
        q.put((rank, "ok", tmax, agg))
    except Exception as e:  # report instead of hanging the test
        q.put((rank, "error", type(e).__name__, str(e)[:200]))


def _run(world, fail_rank=-1, timeout=60):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    out = []
    for _ in range(world):
        out.append(q.get(timeout=timeout))
    for p in procs:
        p.join(timeout=timeout)
        if p.is_alive():
            p.kill()
    return sorted(out)


def test_two_replicas_max_time_and_aggregate():
    res = _run(2)
    assert [r[1] for r in res] == ["ok", "ok"]
    for rank, _, tmax, agg in res:
        assert tmax == 2.0                      # max over ranks
        assert agg == pytest.approx(2 * 100.0 / 2.0)  # all ranks' work over the slowest rank's time


def test_failed_rank_is_reported_not_hung():
    res = _run(2, fail_rank=1, timeout=90)
    status = {r[0]: r[1] for r in res}
    assert status[1] == "error"
    assert status[0] == "error"  # the surviving rank's collective ends with an error (timeout), not a hang


def test_single_process_is_world_one():
    from darray_optimizer_b200 import replicas
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        os.environ.pop(k, None)
    r = replicas.init()
    assert (r.world, r.rank) == (1, 0)
    assert replicas.all_max(r, 3.5) == 3.5
    assert replicas.whole_job_throughput(r, 10.0, 2.0) == 5.0
