"""Pin the FP64 oracle against the reference itself: fixtures in tests/golden/reference_goldens.npz were made by
running the reference's own C++ (compiled from its sources at one MPI rank, oracle/build_ref.sh) through
tests/golden/gen_reference_goldens.py.  The reference computes in FP32 for the dense factorisations and in FP64
for the barrier functions, so tolerances are set per precision."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

G = np.load(Path(__file__).resolve().parent / "golden" / "reference_goldens.npz")


def rel(a, b):
    return np.linalg.norm(np.asarray(a, float) - np.asarray(b, float)) / np.linalg.norm(np.asarray(b, float))


def test_cholesky_known_answer_min_matrix():
    # perftests/perftest_cholesky.cpp:46-53,76-84: chol(min(i+1, j+1)) is the all-ones upper triangle.
    A = G["chol_min_A"]
    R = O.cholesky_upper(A)
    ones = np.triu(np.ones_like(R))
    assert np.max(np.abs(R - ones)) < 1e-12
    for key in ("chol_min_R_blocked", "chol_min_R_recursive"):
        assert np.max(np.abs(G[key] - ones)) < 1e-4  # the reference in FP32
        assert np.max(np.abs(G[key] - R)) < 1e-4


def test_cholesky_test3_factor():
    # tests/test3.cpp:24-46: A = m m^T with m lower triangular (1+i+j) -> upper factor m^T.
    A = G["chol_test3_A"]
    n = A.shape[0]
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    m = np.where(i >= j, 1 + i + j, 0).astype(float)
    assert np.allclose(O.cholesky_upper(A), m.T, rtol=1e-10, atol=1e-10)
    assert rel(G["chol_test3_R"], m.T) < 1e-5


def test_cholesky_random_spd_matches_reference():
    R = O.cholesky_upper(G["chol_spd_A"])
    assert rel(G["chol_spd_R_blocked"], R) < 1e-5


def test_tsqr_matches_reference():
    A = G["tsqr_A"].astype(float)
    Q, R = O.householder_qr(A)
    # LAPACK geqrf conventions match the reference's sgeqrf: same signs, up to FP32 rounding.
    Qs, Rs = O.sign_fix(Q, R)
    Qr, Rr = O.sign_fix(G["tsqr_Q"].astype(float), G["tsqr_R"].astype(float))
    assert rel(Qr, Qs) < 1e-5 and rel(Rr, Rs) < 1e-5
    # CholeskyQR2 spans the same subspace with the same R (positive diagonal)
    Qc, Rc = O.cholqr2(A)
    assert rel(Qc, Qs) < 1e-10 and rel(Rc, Rs) < 1e-10
    assert np.allclose(Qc.T @ Qc, np.eye(A.shape[1]), atol=1e-13)


def test_svd_values_match_reference():
    assert rel(G["svd_S"], O.svd_values(G["svd_A"])) < 1e-5


def test_triangular_solve_matches_reference():
    X = O.trsm_lutn(G["trsm_U"], G["trsm_B"])
    assert rel(G["trsm_X"], X) < 1e-5


def test_matrix_multiply_tn_matches_reference():
    out = O.matmul_tn(G["mm_A"], G["mm_B"], G["mm_C"], alpha=-1.0, beta=1.0)
    assert rel(G["mm_out"], out) < 1e-5


def test_barrier_functions_match_reference_exactly():
    Z, a = G["bar_Z"], G["bar_a"]
    C, t = G["bar_C_t"]
    assert O.f(a, Z) == pytest.approx(float(G["bar_f"][0]), rel=1e-12)
    assert O.gg(a, Z, C, t) == pytest.approx(float(G["bar_gg"][0]), rel=1e-12)
    gf = O.grad_f(Z, a)
    gp = O.grad_phi(a, C, t)
    assert np.allclose(gf, G["bar_grad_f"], rtol=1e-12, atol=1e-13)
    assert np.allclose(gp, G["bar_grad_phi"], rtol=1e-13, atol=0)
    assert np.allclose(O.grad(gf, gp), G["bar_grad"], rtol=1e-12, atol=1e-13)
    assert np.allclose(O.hess_phi(a, C, t), G["bar_D"], rtol=1e-13, atol=0)


def test_pre_conjgrad_matches_reference():
    x, it = O.pre_conjgrad(G["pcg_Z"], G["pcg_M"], G["pcg_D"], G["pcg_b"], G["pcg_a"])
    assert it > 0
    assert rel(x, G["pcg_x"]) < 1e-10


def test_writemodel_text_matches_reference(tmp_path):
    X, y, a, Z = G["wm_X"], G["wm_y"], G["wm_a"], G["wm_Z"]
    res = O.writemodel(tmp_path / "m", a, 1.0, Z, y, X, 0.25, int(np.sum(y == -1)), int(np.sum(y == 1)))
    ref = bytes(G["wm_text"]).decode()
    mine = (tmp_path / "m").read_text()
    assert mine == ref, (mine[:400], ref[:400])
    assert res["nSV"] == int(ref.split("total_sv ")[1].split()[0])


def test_newton_smw_solves_the_newton_system():
    g = np.random.default_rng(0)
    Z = g.standard_normal((400, 12))
    D = g.uniform(1e-3, 1e3, 400)
    r = g.standard_normal(400)
    s = O.newton_smw(Z, D, r)
    H = Z @ Z.T + np.diag(D)
    assert np.allclose(H @ s, -r, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("C", [0.5, 4.0])
def test_barrier_bias_matches_sklearn_svc(C):
    """The oracle's SVM with a bias (dual constraint y^T a = 0, bordered Woodbury Newton steps) against an
    independent solver: scikit-learn's SVC (libsvm SMO) on the same kernel Q = Z Z^T (labels unfolded).  Same dual
    objective to 1e-6 relative, same bias to 1e-5, y^T a = 0 to round-off."""
    from sklearn.svm import SVC
    g = np.random.default_rng(1)
    n, d = 400, 5
    y = np.where(g.random(n) < 0.35, 1.0, -1.0)
    X = g.standard_normal((n, d)) + 0.7 * y[:, None]
    K = O.rbf_block(X, X, None, None, 0.3)
    Q = y[:, None] * K * y[None, :]
    ev, V = np.linalg.eigh(Q)
    keep = ev > 1e-10 * ev.max()
    Z = V[:, keep] * np.sqrt(ev[keep])
    res = O.svm_barrier(Z, y, C, bias=True)
    clf = SVC(C=C, kernel="precomputed", tol=1e-8).fit(y[:, None] * (Z @ Z.T) * y[None, :], y)
    a_sk = np.zeros(n)
    a_sk[clf.support_] = np.abs(clf.dual_coef_[0])
    assert res.status == "converged"
    assert abs(res.f - O.f(a_sk, Z)) <= 1e-6 * abs(res.f)
    assert abs(res.b - clf.intercept_[0]) <= 1e-5
    assert abs(float(y @ res.a)) <= 1e-10 * float(res.a.sum())
    assert res.gap_primal_dual < 1e-6
