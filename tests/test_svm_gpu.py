"""The SVM path on the GPU (through the C ABI) against the FP64 oracle.

* db200_svm_barrier on the oracle's own low-rank factor Z: both run the same FP64 barrier method, so the dual
  objective agrees to relative 1e-9 and both reach the 1e-6 duality-gap stop.
* db200_lowrank: the factor built from bf16 kernel passes vs the oracle's FP64 factor:
  ||Z Z^T - Zo Zo^T||_F <= 2e-2 ||Zo Zo^T||_F.
* db200_svm_solve end to end (config-1 workload): dual objective within 1e-2 of the oracle's, primal-dual gap
  <= 1e-6, held-out accuracy within 1 percentage point.
"""
import numpy as np
import pytest

from darray_optimizer_b200 import datagen
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def dev(a, dtype):
    import torch
    a = np.asarray(a, dtype)
    if a.ndim == 2:
        return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()  # column major
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def zzt_rel(Z, W):
    """||Z Z^T - W W^T||_F / ||W W^T||_F without forming n x n matrices."""
    zz = np.linalg.norm(Z.T @ Z) ** 2
    ww = np.linalg.norm(W.T @ W) ** 2
    zw = np.linalg.norm(Z.T @ W) ** 2
    return np.sqrt(max(zz + ww - 2 * zw, 0.0) / ww)


@pytest.fixture(scope="module")
def c1_small():
    w = datagen.two_gaussians(n=2048, d=16, seed=4)
    w.rank, w.oversample = 48, 8
    lr = O.low_rank_factor(w.X, w.y, w.omega(), w.gamma, w.power_iters)
    return w, lr


def test_barrier_matches_oracle_on_same_factor(gpu_ctx, c1_small):
    import torch
    w, lr = c1_small
    n, r = lr.Z.shape
    ref = O.svm_barrier(lr.Z, w.y, w.C)
    dZ, dy = dev(lr.Z, np.float64), dev(w.y, np.float32)
    da = torch.zeros(n, dtype=torch.float64, device="cuda")
    rep = gpu_ctx.svm_barrier(n, r, dZ.data_ptr(), n, dy.data_ptr(), w.C, da.data_ptr())
    a = da.cpu().numpy()
    assert rep.status == 0
    assert abs(rep.f - ref.f) <= 1e-9 * abs(ref.f)
    assert abs(O.f(a, lr.Z) - ref.f) <= 1e-9 * abs(ref.f)
    assert rep.outer == ref.outer
    assert abs(rep.newton - ref.newton) <= 2
    assert rep.gap_barrier < 1e-6 and ref.gap_barrier < 1e-6
    assert rep.gap_primal_dual < 1e-6
    assert np.all(a > 0) and np.all(a < w.C)
    assert np.max(np.abs(a - ref.a)) <= 1e-6 * w.C


def test_barrier_iteration_caps_report_maxiter(gpu_ctx, c1_small):
    import torch
    w, lr = c1_small
    n, r = lr.Z.shape
    dZ, dy = dev(lr.Z, np.float64), dev(w.y, np.float32)
    da = torch.zeros(n, dtype=torch.float64, device="cuda")
    p = gpu_ctx.barrier_params(max_outer=2)
    rep = gpu_ctx.svm_barrier(n, r, dZ.data_ptr(), n, dy.data_ptr(), w.C, da.data_ptr(), params=p,
                              allow_maxiter=True)
    assert rep.status == -4 and rep.outer == 2  # DB200_ERR_MAXITER


def test_lowrank_factor_matches_oracle(gpu_ctx):
    import torch
    w = datagen.two_gaussians(n=4096, d=32, seed=1)
    Om = w.omega()
    lr = O.low_rank_factor(w.X, w.y, Om, w.gamma, w.power_iters)
    n, l = w.n, w.l
    dX, dy, dO = dev(w.X.T, np.float32), dev(w.y, np.float32), dev(Om, np.float32)  # X point-major = d x n col
    dZ = torch.zeros((l, n), dtype=torch.float64, device="cuda")
    rep = gpu_ctx.lowrank(n, w.d, l, w.power_iters, dX.data_ptr(), w.d, dy.data_ptr(), dO.data_ptr(), n, w.gamma,
                          dZ.data_ptr(), n)
    Z = dZ.cpu().numpy().T
    assert zzt_rel(Z, lr.Z) <= 2e-2
    assert rep.nu > 0


def test_svm_solve_end_to_end_matches_oracle(gpu_ctx):
    import torch
    w = datagen.two_gaussians(n=4096, d=32, seed=1)
    test = datagen.two_gaussians(n=2048, d=32, seed=2)
    Om = w.omega()
    lr = O.low_rank_factor(w.X, w.y, Om, w.gamma, w.power_iters)
    ref = O.svm_barrier(lr.Z, w.y, w.C)
    n, l = w.n, w.l
    dX, dy, dO = dev(w.X.T, np.float32), dev(w.y, np.float32), dev(Om, np.float32)
    dZ = torch.zeros((l, n), dtype=torch.float64, device="cuda")
    da = torch.zeros(n, dtype=torch.float64, device="cuda")
    rep = gpu_ctx.svm_solve(n, w.d, l, w.power_iters, dX.data_ptr(), w.d, dy.data_ptr(), dO.data_ptr(), n,
                            w.gamma, w.C, da.data_ptr(), dZ.data_ptr(), n)
    a = da.cpu().numpy()
    assert rep.status == 0
    assert rep.gap_barrier < 1e-6 and rep.gap_primal_dual < 1e-6
    assert abs(rep.f - ref.f) <= 1e-2 * abs(ref.f)
    acc_gpu = np.mean(np.sign(O.decision(test.X, w.X, w.y, a, w.gamma)) == test.y)
    acc_ref = np.mean(np.sign(O.decision(test.X, w.X, w.y, ref.a, w.gamma)) == test.y)
    assert abs(acc_gpu - acc_ref) <= 0.01
    assert rep.ms_total > 0 and rep.ms_sketch > 0
