"""db200_rbf_sketch_noalloc: the allocation-free fused RBF x sketch, for callers that cannot call cudaMalloc
(plugin hosts that own every device allocation and only lend a stream, hard memory budgets, phases that must not
enter the allocator).  It uses one fixed static device scratch array instead of a workspace.

Checked through the C ABI against the allocating entry point db200_rbf_sketch, on two calls in a row (the
scratch keeps the previous call's contents, so the second call must not depend on it), within relative Frobenius
error 2e-3 (TOL, the single fp16 sketch product's tolerance in tests/test_rbf_gpu.py; both paths share the
kernels, so the measured difference is at the level of fp32 summation order).  Also: point- and feature-major
inputs, Xi == Xj and Xi != Xj, n = 0 (Y = 0), argument errors, requests beyond the scratch, and that a call after
warm-up leaves the device's free memory unchanged.  This file sorts last so that a run stopping at its first
failure has already run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from darray_optimizer_b200 import _lib
from util import colmajor_empty, colmajor_host, dev, ptr, rel_fro

pytestmark = pytest.mark.gpu

POINT_MAJOR, FEATURE_MAJOR = 0, 1
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


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("layout", [POINT_MAJOR, FEATURE_MAJOR])
def test_noalloc_matches_allocating_sketch_twice(gpu_ctx, layout):
    lib = _lib.load()
    cases = [(3, 2048, 2048, 64, 200), (4, 777, 1500, 33, 528)]  # (seed, m, n, d, l); second: Xi != Xj
    for seed, m, n, d, l in cases:
        Xi, Xj, yi, yj, Om = _case(seed, n, d, l, m)
        if layout == POINT_MAJOR:
            dXi = dev(Xi)
            dXj = dXi if Xj is Xi else dev(Xj)
            ldxi, ldxj = d, d
        else:  # m x d column major: the transposed bytes
            dXi = dev(np.asfortranarray(Xi))
            dXj = dXi if Xj is Xi else dev(np.asfortranarray(Xj))
            ldxi, ldxj = m, n
        dyi = dev(yi)
        dyj = dyi if yj is yi else dev(yj)
        dOm = dev(np.asfortranarray(Om))
        gamma = 1.0 / d
        Yref = colmajor_empty(m, l)
        gpu_ctx.rbf_sketch(m, n, d, l, ptr(dXi), ldxi, ptr(dXj), ldxj, layout, ptr(dyi), ptr(dyj), ptr(dOm), n,
                           ptr(Yref), m, gamma)
        gpu_ctx.sync()
        ref = colmajor_host(Yref, m)
        for call in range(2):  # two calls in a row on the shared scratch
            Y = colmajor_empty(m, l)
            st = lib.db200_rbf_sketch_noalloc(_stream(), m, n, d, l, ptr(dXi), ldxi, ptr(dXj), ldxj, layout,
                                              ptr(dyi), ptr(dyj), ptr(dOm), n, ptr(Y), m, gamma)
            assert st == 0, (call, _lib.STATUS.get(st, st))
            got = colmajor_host(Y, m)
            assert rel_fro(got, ref) <= TOL, (seed, call)


def test_noalloc_leaves_free_memory_unchanged(gpu_ctx):
    """After a warm-up call (which loads the library's kernels into the context), further calls change the
    device's free memory by nothing: no allocation behind the caller's back."""
    import torch
    lib = _lib.load()
    m = n = 4096
    d, l = 32, 64
    Xi, _, yi, _, Om = _case(8, n, d, l)
    dX, dy, dOm = dev(Xi), dev(yi), dev(np.asfortranarray(Om))
    Y = colmajor_empty(m, l)
    args = (m, n, d, l, ptr(dX), d, ptr(dX), d, POINT_MAJOR, ptr(dy), ptr(dy), ptr(dOm), n, ptr(Y), m, 1.0 / d)
    assert lib.db200_rbf_sketch_noalloc(_stream(), *args) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert lib.db200_rbf_sketch_noalloc(_stream(), *args) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_empty_columns_and_argument_errors(gpu_ctx):
    import torch
    lib = _lib.load()
    m, d, l = 300, 16, 24
    X = torch.ones((m, d), dtype=torch.float32, device="cuda")
    O = torch.ones((l, m), dtype=torch.float32, device="cuda")
    # n = 0: an empty sum, Y = 0 as db200_rbf_sketch gives (Y starts as ones here)
    Y = torch.ones((l, m + 5), dtype=torch.float32, device="cuda")
    st = lib.db200_rbf_sketch_noalloc(_stream(), m, 0, d, l, X.data_ptr(), d, X.data_ptr(), d, POINT_MAJOR, 0, 0,
                                      O.data_ptr(), 1, Y.data_ptr(), m + 5, 0.5)
    assert st == 0
    Yh = Y.cpu().numpy()
    assert np.all(Yh[:, :m] == 0.0) and np.all(Yh[:, m:] == 1.0)  # the padding rows past m are not touched
    Y = torch.zeros((l, m), dtype=torch.float32, device="cuda")
    base = dict(stream=_stream(), m=m, n=m, d=d, l=l, Xi=X.data_ptr(), ldxi=d, Xj=X.data_ptr(), ldxj=d,
                layout=POINT_MAJOR, yi=0, yj=0, Om=O.data_ptr(), ldo=m, Y=Y.data_ptr(), ldy=m, gamma=0.5)
    for bad in (dict(ldy=m - 1), dict(ldo=m - 1), dict(ldxi=d - 1), dict(layout=7), dict(d=0), dict(Om=0),
                dict(m=-1)):
        a = dict(base, **bad)
        st = lib.db200_rbf_sketch_noalloc(*a.values())
        assert st == -1, (bad, _lib.STATUS.get(st, st))  # DB200_ERR_INVALID
    a = dict(base, d=129, ldxi=129, ldxj=129)  # beyond the kernels' feature width: refused before any access
    assert lib.db200_rbf_sketch_noalloc(*a.values()) == -8  # DB200_ERR_UNSUPPORTED


def test_noalloc_rejects_requests_beyond_its_scratch(gpu_ctx):
    import torch
    lib = _lib.load()
    # n = 300000 points of d = 8: the packed points alone need ~38 MB > the 32 MiB array.  Real buffers of the
    # stated sizes are passed so that nothing could be read out of bounds even if the check were missing.
    n, d, l = 300000, 8, 16
    X = torch.zeros((n, d), dtype=torch.float32, device="cuda")
    O = torch.zeros((l, n), dtype=torch.float32, device="cuda")
    Y = torch.zeros((l, n), dtype=torch.float32, device="cuda")
    st = lib.db200_rbf_sketch_noalloc(_stream(), n, n, d, l, X.data_ptr(), d, X.data_ptr(), d, POINT_MAJOR, 0, 0,
                                      O.data_ptr(), n, Y.data_ptr(), n, 0.1)
    assert st == -9  # DB200_ERR_TOO_LARGE
