"""The SVM path on the GPU (through the C ABI) against the FP64 oracle.

* db200_svm_barrier on the oracle's own low-rank factor Z: both run the same FP64 barrier method, so the dual
  objective agrees to relative 1e-9 and both reach the 1e-6 duality-gap stop.
* db200_lowrank: the factor built from tensor-core kernel passes vs the oracle's FP64 factor,
  ||Z Z^T - Zo Zo^T||_F / ||Zo Zo^T||_F: <= 1e-5 with the compensated sketch product (DB200_MIXED),
  <= 2e-2 with the single fp16 product (DB200_MIXED_FAST).
* db200_svm_solve end to end on the two-Gaussian workload (n = 4096, d = 32, l = 138, q = 1, C = 1): dual
  objective within 1e-6 of the oracle's (DB200_MIXED and DB200_FP64; the fast mixed form, whose single fp16 sketch
  product moves the sketched subspace, within 1e-4), primal-dual gap <= 1e-6, held-out accuracy within 1
  percentage point.
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


@pytest.mark.parametrize("precision", [0, 1])  # DB200_MIXED (tensor-core capacity matrix + refinement), DB200_FP64
def test_barrier_matches_oracle_on_same_factor(gpu_ctx, c1_small, precision):
    import torch
    w, lr = c1_small
    n, r = lr.Z.shape
    ref = O.svm_barrier(lr.Z, w.y, w.C)
    dZ, dy = dev(lr.Z, np.float64), dev(w.y, np.float32)
    da = torch.zeros(n, dtype=torch.float64, device="cuda")
    p = gpu_ctx.barrier_params(precision=precision)
    rep = gpu_ctx.svm_barrier(n, r, dZ.data_ptr(), n, dy.data_ptr(), w.C, da.data_ptr(), params=p)
    if precision == 0:
        # the int8 (Ozaki) capacity matrix is accurate enough that no Newton step falls back to the FP64 one
        assert rep.fallbacks == 0
    a = da.cpu().numpy()
    assert rep.status == 0
    tol = 1e-9 if precision == 1 else 1e-8  # mixed: Newton steps refined to relative residual 1e-10
    assert abs(rep.f - ref.f) <= tol * abs(ref.f)
    assert abs(O.f(a, lr.Z) - ref.f) <= tol * abs(ref.f)
    assert rep.outer == ref.outer
    assert abs(rep.newton - ref.newton) <= 2
    assert rep.gap_barrier < 1e-6 and ref.gap_barrier < 1e-6
    assert rep.gap_primal_dual < 1e-6
    assert np.all(a > 0) and np.all(a < w.C)
    assert np.max(np.abs(a - ref.a)) <= 1e-6 * w.C


@pytest.mark.parametrize("precision", [0, 1])
def test_barrier_bias_matches_oracle(gpu_ctx, c1_small, precision):
    """The SVM with a bias (the dual's y^T a = 0, bordered Woodbury Newton steps) against the oracle's, which
    tests/test_oracle.py checks against scikit-learn's SVC: same objective and bias, y^T a = 0 kept."""
    import torch
    w, lr = c1_small
    n, r = lr.Z.shape
    ref = O.svm_barrier(lr.Z, w.y, w.C, bias=True)
    dZ, dy = dev(lr.Z, np.float64), dev(w.y, np.float32)
    da = torch.zeros(n, dtype=torch.float64, device="cuda")
    p = gpu_ctx.barrier_params(precision=precision, bias=1)
    rep = gpu_ctx.svm_barrier(n, r, dZ.data_ptr(), n, dy.data_ptr(), w.C, da.data_ptr(), params=p)
    a = da.cpu().numpy()
    assert rep.status == 0
    tol = 1e-9 if precision == 1 else 1e-8
    assert abs(rep.f - ref.f) <= tol * abs(ref.f)
    assert abs(rep.b - ref.b) <= 1e-6 * max(1.0, abs(ref.b))
    assert abs(float(w.y.astype(np.float64) @ a)) <= 1e-10 * float(a.sum())
    assert rep.gap_barrier < 1e-6 and rep.gap_primal_dual < 1e-6
    assert np.all(a > 0) and np.all(a < w.C)
    assert np.max(np.abs(a - ref.a)) <= 1e-6 * w.C
    # the bias changes the solution: the no-bias dual reaches a lower objective (fewer constraints)
    nob = O.svm_barrier(lr.Z, w.y, w.C)
    assert nob.f <= ref.f


def test_barrier_bias_needs_both_classes(gpu_ctx, c1_small):
    import torch
    from darray_optimizer_b200._lib import DB200Error
    w, lr = c1_small
    n, r = lr.Z.shape
    dZ, dy = dev(lr.Z, np.float64), dev(np.ones(n, np.float32), np.float32)
    da = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(DB200Error) as e:
        gpu_ctx.svm_barrier(n, r, dZ.data_ptr(), n, dy.data_ptr(), w.C, da.data_ptr(),
                            params=gpu_ctx.barrier_params(bias=1))
    assert e.value.status == -5  # DB200_ERR_INFEASIBLE


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


@pytest.mark.parametrize("precision,tol", [(0, 1e-5), (2, 2e-2), (1, 1e-9)])
def test_lowrank_factor_matches_oracle(gpu_ctx, precision, tol):
    """DB200_MIXED (compensated sketch product): ||ZZ^T - ZoZo^T|| <= 1e-5; DB200_MIXED_FAST (single fp16
    product): <= 2e-2.  FP64 comparator: the oracle's own algorithm in FP64, <= 1e-9 (the shifted Cholesky and
    CholeskyQR2 run in the same order)."""
    import torch
    w = datagen.two_gaussians(n=4096, d=32, seed=1)
    Om = w.omega()
    lr = O.low_rank_factor(w.X, w.y, Om, w.gamma, w.power_iters)
    n, l = w.n, w.l
    dX, dy, dO = dev(w.X.T, np.float32), dev(w.y, np.float32), dev(Om, np.float32)  # X point-major = d x n col
    dZ = torch.zeros((l, n), dtype=torch.float64, device="cuda")
    rep = gpu_ctx.lowrank(n, w.d, l, w.power_iters, dX.data_ptr(), w.d, dy.data_ptr(), dO.data_ptr(), n, w.gamma,
                          dZ.data_ptr(), n, precision=precision)
    Z = dZ.cpu().numpy().T
    if precision == 1:  # same FP64 algorithm: compare the factor itself (the identity below cancels at ~1e-8)
        assert np.linalg.norm(Z - lr.Z) <= tol * np.linalg.norm(lr.Z)
    else:
        err = zzt_rel(Z, lr.Z)
        print(f"lowrank precision={precision}: ||ZZ^T - ZoZo^T||/||ZoZo^T|| = {err:.3e}")
        assert err <= tol
    assert rep.nu > 0


# dual objective against the oracle's: 1e-6 relative (the SVM parity target) for the compensated mixed path and FP64; the fast
# mixed form's single fp16 sketch product leaves ~2e-5 at this size (4e-4 at n = 131072)
@pytest.mark.parametrize("precision,ftol", [(0, 1e-6), (1, 1e-8), (2, 1e-4)])
def test_svm_solve_end_to_end_matches_oracle(gpu_ctx, precision, ftol):
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
                            w.gamma, w.C, da.data_ptr(), dZ.data_ptr(), n,
                            params=gpu_ctx.barrier_params(precision=precision))
    a = da.cpu().numpy()
    assert rep.status == 0
    assert rep.gap_barrier < 1e-6 and rep.gap_primal_dual < 1e-6
    rel = abs(rep.f - ref.f) / abs(ref.f)
    print(f"svm_solve precision={precision}: |f - f_oracle|/|f_oracle| = {rel:.3e}")
    assert rel <= ftol
    acc_gpu = np.mean(np.sign(O.decision(test.X, w.X, w.y, a, w.gamma)) == test.y)
    acc_ref = np.mean(np.sign(O.decision(test.X, w.X, w.y, ref.a, w.gamma)) == test.y)
    assert abs(acc_gpu - acc_ref) <= 0.01
    assert rep.ms_total > 0 and rep.ms_sketch > 0


def test_barrier_terms_match_reference_goldens(gpu_ctx):
    # include/dbarrier.h:14-81 run by the reference itself (tests/golden): f, gg, Grad_f, Grad_Phi, Grad, Hess_Phi
    import torch
    from pathlib import Path
    G = np.load(Path(__file__).resolve().parent / "golden" / "reference_goldens.npz")
    Z, a = G["bar_Z"], G["bar_a"]
    C, t = G["bar_C_t"]
    n, k = Z.shape
    dZ, da = dev(Z, np.float64), dev(a, np.float64)
    outs = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(4)]
    f, gg = gpu_ctx.barrier_terms(n, k, dZ.data_ptr(), n, da.data_ptr(), C, t, *[o.data_ptr() for o in outs])
    gf, gp, gr, D = (o.cpu().numpy() for o in outs)
    assert f == pytest.approx(float(G["bar_f"][0]), rel=1e-12)
    assert gg == pytest.approx(float(G["bar_gg"][0]), rel=1e-12)
    assert np.allclose(gf, G["bar_grad_f"], rtol=1e-12, atol=1e-13)
    assert np.allclose(gp, G["bar_grad_phi"], rtol=1e-13, atol=0)
    assert np.allclose(gr, G["bar_grad"], rtol=1e-12, atol=1e-13)
    assert np.allclose(D, G["bar_D"], rtol=1e-13, atol=0)


def test_woodbury_solve_matches_dense_solve(gpu_ctx):
    import torch
    g = np.random.default_rng(2)
    n, r = 3000, 40
    Z = g.standard_normal((n, r))
    diag = np.exp(g.uniform(-8, 8, n))  # dynamic range like the barrier's D late in the solve
    b = g.standard_normal(n)
    dZ, dd, db = dev(Z, np.float64), dev(diag, np.float64), dev(b, np.float64)
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    gpu_ctx.woodbury_solve(n, r, dZ.data_ptr(), n, dd.data_ptr(), db.data_ptr(), dx.data_ptr())
    x = dx.cpu().numpy()
    H = Z @ Z.T + np.diag(diag)
    assert np.linalg.norm(H @ x - b) <= 1e-9 * np.linalg.norm(b) * (1 + np.linalg.norm(H, 2) * np.linalg.norm(x) /
                                                                     np.linalg.norm(b))
    # same system pinned through the oracle's pre_conjgrad fixture: exact solve has residual far below 1e-2
    from pathlib import Path
    G = np.load(Path(__file__).resolve().parent / "golden" / "reference_goldens.npz")
    Zp, Dp, bp = G["pcg_Z"], G["pcg_D"], G["pcg_b"]
    npc, kpc = Zp.shape
    dz2, dd2, db2 = dev(Zp, np.float64), dev(Dp + npc, np.float64), dev(bp, np.float64)
    dx2 = torch.zeros(npc, dtype=torch.float64, device="cuda")
    gpu_ctx.woodbury_solve(npc, kpc, dz2.data_ptr(), npc, dd2.data_ptr(), db2.data_ptr(), dx2.data_ptr())
    x2 = dx2.cpu().numpy()
    A = Zp @ Zp.T + np.diag(Dp + npc)
    assert np.linalg.norm(A @ x2 - bp) < 1e-12
    assert np.linalg.norm(A @ G["pcg_x"] - bp) <= 1e-2  # the reference's PCG stopping rule


@pytest.mark.parametrize("r", [1, 31, 33, 97, 528, 1040, 2064])
def test_woodbury_solve_ragged_and_large_rank(gpu_ctx, r):
    # every shape of the 32-row triangular-solve blocks (partial last block, one block, many) and of the 64-column
    # Cholesky block columns, against a dense FP64 solve of the same system
    import torch
    g = np.random.default_rng(r)
    n = max(2 * r, 256)
    Z = g.standard_normal((n, r)) / np.sqrt(r)
    diag = np.exp(g.uniform(-3, 3, n))
    b = g.standard_normal(n)
    dZ, dd, db = dev(Z, np.float64), dev(diag, np.float64), dev(b, np.float64)
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    gpu_ctx.woodbury_solve(n, r, dZ.data_ptr(), n, dd.data_ptr(), db.data_ptr(), dx.data_ptr())
    x = dx.cpu().numpy()
    H = Z @ Z.T + np.diag(diag)
    x_ref = np.linalg.solve(H, b)
    assert np.linalg.norm(x - x_ref) <= 1e-10 * np.linalg.norm(x_ref)


def test_knorm_matches_oracle(gpu_ctx, c1_small):
    w, lr = c1_small
    n, k = lr.Z.shape
    dX, dy, dZ = dev(w.X.T, np.float32), dev(w.y, np.float32), dev(lr.Z, np.float64)
    kn, rn, ratio = gpu_ctx.knorm(n, w.d, k, dX.data_ptr(), w.d, dy.data_ptr(), dZ.data_ptr(), n, w.gamma)
    okn, orn, oratio = O.knorm(w.X, w.y, lr.Z, w.gamma)
    assert kn == pytest.approx(okn, rel=1e-5)
    assert rn == pytest.approx(orn, rel=1e-3)
    assert ratio == pytest.approx(oratio, rel=1e-3)
