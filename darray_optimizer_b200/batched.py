"""Batched SVM workload: many independent instances of uneven size and hyperparameters solved together
(db200_svm_solve_batched), with tile plans from the autotuner.

The workload: `count` instances with n log-uniform in [2048, 65536], d drawn from {16, 64, 128}, data from the
two-Gaussians or the uniform-hyperplane generator (alternating, per-instance seeds), hyperparameters on an 8 x 8
grid gamma in {2^-6 .. 2^1} / d and C in {2^-2 .. 2^5}, rank r = min(256, n / 16) plus 16 oversampling columns and
one power iteration.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import datagen


def workload(count: int = 64, seed: int = 4):
    g = datagen.rng(seed)
    out = []
    for k in range(count):
        n = int(round(math.exp(g.uniform(math.log(2048), math.log(65536)))))
        d = int(g.choice([16, 64, 128]))
        gen = "two_gaussians" if k % 2 == 0 else "uniform_hyperplane"
        gi, ci = k % 8, (k // 8) % 8
        gamma = 2.0 ** (gi - 6) / d
        C = 2.0 ** (ci - 2)
        r = min(256, n // 16)
        out.append({"k": k, "n": n, "d": d, "gen": gen, "gamma": gamma, "C": C, "r": r, "l": r + 16,
                    "seed": 1000 + k})
    return out


def materialise(spec):
    """(X, y, Omega) host arrays of one instance."""
    if spec["gen"] == "two_gaussians":
        w = datagen.two_gaussians(n=spec["n"], d=spec["d"], seed=spec["seed"])
    else:
        w = datagen.uniform_hyperplane(n=spec["n"], d=spec["d"], seed=spec["seed"])
    Om = datagen.rng(spec["seed"] + 7919).standard_normal((spec["n"], spec["l"]), dtype=np.float32)
    return w.X, w.y, Om


def upload(specs):
    """Device buffers of every instance (kept alive by the returned list)."""
    import torch
    bufs = []
    for s in specs:
        X, y, Om = materialise(s)
        bufs.append({"X": torch.from_numpy(X).cuda(), "y": torch.from_numpy(y).cuda(),
                     "Om": torch.from_numpy(np.ascontiguousarray(Om.T)).cuda(),
                     "Z": torch.empty((s["l"], s["n"]), dtype=torch.float64, device="cuda"),
                     "a": torch.empty(s["n"], dtype=torch.float64, device="cuda")})
    return bufs


def solve_batched(ctx, specs, bufs, tuner=None, use_graph=True, workers=8, q=1):
    """One db200_svm_solve_batched call; returns (wall seconds, per-instance reports, batch report, plans)."""
    import torch
    from ._lib import SvmInstance
    plans = []
    inst = []
    for s, b in zip(specs, bufs):
        plan = tuner.plan(s["n"], s["d"], s["l"]) if tuner else (0, 0, 0)
        plans.append(plan)
        inst.append(SvmInstance(s["n"], s["d"], s["l"], b["X"].data_ptr(), s["d"], b["y"].data_ptr(), s["gamma"],
                                s["C"], b["Om"].data_ptr(), s["n"], b["Z"].data_ptr(), s["n"], b["a"].data_ptr(),
                                *plan))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    reps, brep = ctx.svm_solve_batched(inst, q=q, use_graph=use_graph, workers=workers)
    torch.cuda.synchronize()
    return time.perf_counter() - t0, reps, brep, plans


def solve_sequential(ctx, specs, bufs, q=1):
    """The same instances one after another through the single-problem path (db200_svm_solve)."""
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    reps = []
    for s, b in zip(specs, bufs):
        reps.append(ctx.svm_solve(s["n"], s["d"], s["l"], q, b["X"].data_ptr(), s["d"], b["y"].data_ptr(),
                                  b["Om"].data_ptr(), s["n"], s["gamma"], s["C"], b["a"].data_ptr(),
                                  b["Z"].data_ptr(), s["n"]))
    torch.cuda.synchronize()
    return time.perf_counter() - t0, reps
