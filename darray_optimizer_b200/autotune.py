"""Tile-plan autotuner for the fused RBF x sketch engine.

The tile engine's free shape parameters per problem are the sketch panel plan: how many panels the l sketch
columns are cut into (each pass over the points recomputes the distance tile once per panel), the panel width (a
multiple of 16, at most 320) and how many 128-column distance buffers (1 or 2) share tensor memory with the
panel (panel + 64 + 128 * buffers <= 512 columns).  tune() times every valid plan for a shape on synthetic data of
that shape through db200_rbf_sketch_batched and keeps the fastest; Tuner caches the choice per shape class
(padded feature width, padded sketch width, power-of-two size class of n) in memory and, optionally, in a JSON
file.
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

TMEM_COLS = 512


def candidate_plans(l: int) -> list[tuple[int, int, int]]:
    """Valid (n_panels, panel, g_bufs) plans for sketch width l: the fewest panels each buffer count allows and
    one more."""
    lpad = -(-max(l, 1) // 16) * 16
    out = []
    for g in (1, 2):
        pmax = TMEM_COLS - 64 - 128 * g
        pmax = min(320, pmax - pmax % 16)
        first = -(-lpad // pmax)
        for np_ in (first, first + 1):
            panel = -(-(-(-lpad // np_)) // 16) * 16
            if 16 <= panel <= pmax and np_ * panel >= lpad:
                out.append((np_, panel, g))
    return sorted(set(out))


def shape_key(n: int, d: int, l: int) -> str:
    dp = -(-max(d, 1) // 32) * 32
    lpad = -(-max(l, 1) // 16) * 16
    return f"dp{dp}_l{lpad}_n{int(round(math.log2(max(n, 1))))}"


def tune(ctx, n: int, d: int, l: int, reps: int = 3, seed: int = 0) -> tuple[tuple[int, int, int], dict]:
    """Fastest plan for one (n, d, l) shape and the median milliseconds of every candidate."""
    import torch
    from ._lib import SketchJob
    g = np.random.default_rng(seed)
    X = torch.from_numpy(g.random((n, d), dtype=np.float32)).cuda()
    y = torch.from_numpy(np.where(g.random(n) < 0.5, 1.0, -1.0).astype(np.float32)).cuda()
    Om = torch.from_numpy(g.standard_normal((l, n), dtype=np.float32)).cuda()  # n x l column major
    Y = torch.empty((l, n), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    times = {}
    for plan in candidate_plans(l):
        job = SketchJob(n, n, d, l, X.data_ptr(), d, X.data_ptr(), d, y.data_ptr(), y.data_ptr(), Om.data_ptr(), n,
                        Y.data_ptr(), n, 1.0 / d, *plan)
        ctx.rbf_sketch_batched([job])  # warm-up (module load, workspace growth)
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.rbf_sketch_batched([job])
            e1.record(stream)
            ctx.sync()
            ms.append(e0.elapsed_time(e1))
        times[plan] = float(np.median(ms))
    best = min(times, key=times.get)
    return best, {f"{p[0]}x{p[1]}/g{p[2]}": t for p, t in times.items()}


class Tuner:
    """Plan cache keyed by shape class; tunes on first sight of a class."""

    def __init__(self, ctx, path: str | Path | None = None):
        self.ctx = ctx
        self.path = Path(path) if path else None
        self.cache: dict[str, dict] = {}
        if self.path and self.path.exists():
            self.cache = json.loads(self.path.read_text())

    def plan(self, n: int, d: int, l: int) -> tuple[int, int, int]:
        key = shape_key(n, d, l)
        if key not in self.cache:
            # tune at the class's representative size (the power of two) so one entry serves the whole class
            n_rep = 2 ** int(round(math.log2(max(n, 256))))
            best, times = tune(self.ctx, n_rep, d, l)
            self.cache[key] = {"plan": list(best), "ms": times, "n_tuned": n_rep}
            if self.path:
                self.path.write_text(json.dumps(self.cache, indent=1, sort_keys=True))
        return tuple(self.cache[key]["plan"])
