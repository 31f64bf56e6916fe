"""db200_rbf_sketch_noalloc: the allocation-free fused RBF x sketch, for callers that cannot call cudaMalloc
(plugin hosts that own every device allocation and only lend a stream, hard memory budgets, phases that must not
enter the allocator).  It uses one fixed static device scratch array instead of a workspace.

Checked through the C ABI against the allocating entry point db200_rbf_sketch, on two calls in a row (the
scratch keeps the previous call's contents, so the second call must not depend on it), within the sketch
tolerance used by tests/test_rbf_gpu.py (relative Frobenius error 1e-2).  This file sorts last so that a run
stopping at its first failure has already run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from darray_optimizer_b200 import _lib
from util import colmajor_empty, colmajor_host, dev, ptr, rel_fro

pytestmark = pytest.mark.gpu

POINT_MAJOR = 0
TOL = 2e-3


def _case(seed, n, d, l, m=None):
    g = np.random.default_rng(seed)
    m = m or n
    Xi = (0.5 * g.standard_normal((m, d))).astype(np.float32)
    Xj = Xi if m == n else (0.5 * g.standard_normal((n, d))).astype(np.float32)
    yi = np.where(g.random(m) < 0.5, 1.0, -1.0).astype(np.float32)
    yj = yi if m == n else np.where(g.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    Om = g.standard_normal((n, l)).astype(np.float32)
    return Xi, Xj, yi, yj, Om


def test_noalloc_matches_allocating_sketch_twice(gpu_ctx):
    import torch
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    cases = [(3, 2048, 2048, 64, 200), (4, 777, 1500, 33, 528)]  # (seed, m, n, d, l); second: Xi != Xj
    for seed, m, n, d, l in cases:
        Xi, Xj, yi, yj, Om = _case(seed, n, d, l, m)
        dXi = dev(Xi)
        dXj = dXi if Xj is Xi else dev(Xj)
        dyi = dev(yi)
        dyj = dyi if yj is yi else dev(yj)
        dOm = dev(np.asfortranarray(Om))
        gamma = 1.0 / d
        Yref = colmajor_empty(m, l)
        gpu_ctx.rbf_sketch(m, n, d, l, ptr(dXi), d, ptr(dXj), d, POINT_MAJOR, ptr(dyi), ptr(dyj), ptr(dOm), n,
                           ptr(Yref), m, gamma)
        gpu_ctx.sync()
        ref = colmajor_host(Yref, m)
        for call in range(2):  # two calls in a row on the shared scratch
            Y = colmajor_empty(m, l)
            st = lib.db200_rbf_sketch_noalloc(stream, m, n, d, l, ptr(dXi), d, ptr(dXj), d, POINT_MAJOR, ptr(dyi),
                                              ptr(dyj), ptr(dOm), n, ptr(Y), m, gamma)
            assert st == 0, (call, _lib.STATUS.get(st, st))
            got = colmajor_host(Y, m)
            assert rel_fro(got, ref) <= TOL, (seed, call)


def test_noalloc_rejects_requests_beyond_its_scratch(gpu_ctx):
    import torch
    lib = _lib.load()
    # n = 300000 points of d = 8: the packed points alone need ~38 MB > the 32 MiB array.  Real buffers of the
    # stated sizes are passed so that nothing could be read out of bounds even if the check were missing.
    n, d, l = 300000, 8, 16
    X = torch.zeros((n, d), dtype=torch.float32, device="cuda")
    O = torch.zeros((l, n), dtype=torch.float32, device="cuda")
    Y = torch.zeros((l, n), dtype=torch.float32, device="cuda")
    st = lib.db200_rbf_sketch_noalloc(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), n, n, d, l,
                                      X.data_ptr(), d, X.data_ptr(), d, POINT_MAJOR, 0, 0, O.data_ptr(), n,
                                      Y.data_ptr(), n, 0.1)
    assert st == -9  # DB200_ERR_TOO_LARGE
