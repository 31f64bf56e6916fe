"""CPU checks of the learned-landmark oracle itself (no GPU): the MLP gradient against central finite
differences, bf16 rounding, k-NN, ridge leverage identities, the Gumbel keys and the exact-Nystrom limit."""
import numpy as np

from oracle import landmarks as LO


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 3.0e38, 1e-40], dtype=np.float32)
    r = LO.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0  # halfway between 1 and 1 + 2^-7: ties to even
    assert r[2] == 1.0 + 2.0 ** -6  # halfway between 1 + 2^-7 and 1 + 2^-6: ties to even (up)
    assert r[3] == -2.5
    assert np.isfinite(r[4])


def test_mlp_gradient_matches_finite_differences():
    g = np.random.default_rng(0)
    in_dim, width, hidden, m = 6, 8, 3, 20
    layout, npar = LO.mlp_layout(in_dim, width, hidden)
    p = g.standard_normal(npar) * 0.4
    F = g.standard_normal((m, in_dim))
    t = g.standard_normal(m)
    mean, scale = F.mean(0), 1.0 / F.std(0)
    loss, grad = LO.mlp_loss_grad(p, F, t, mean, scale, width, hidden, round_bf16=False)
    eps = 1e-6
    fd = np.empty(npar)
    for k in range(npar):
        e = np.zeros(npar)
        e[k] = eps
        lp, _ = LO.mlp_loss_grad(p + e, F, t, mean, scale, width, hidden, round_bf16=False)
        lm, _ = LO.mlp_loss_grad(p - e, F, t, mean, scale, width, hidden, round_bf16=False)
        fd[k] = (lp - lm) / (2 * eps)
    assert np.linalg.norm(fd - grad) <= 1e-6 * np.linalg.norm(fd)
    assert loss > 0


def test_knn_oracle_brute_force():
    g = np.random.default_rng(1)
    X = g.standard_normal((60, 5))
    ref = np.sort(g.choice(60, size=25, replace=False))
    got = LO.knn_distance(X, ref, 3)
    for i in range(60):
        ds = sorted(np.linalg.norm(X[i] - X[j]) for j in ref if j != i)
        assert abs(got[i] - ds[2]) <= 1e-9


def test_ridge_leverage_sums_to_effective_dimension():
    g = np.random.default_rng(2)
    Z = g.standard_normal((200, 12))
    lam = 3.0
    lev = LO.ridge_leverage(Z, lam)
    s = np.linalg.svd(Z, compute_uv=False)
    assert abs(lev.sum() - np.sum(s ** 2 / (s ** 2 + lam))) <= 1e-10
    assert np.all((lev > 0) & (lev < 1))


def test_gumbel_keys_deterministic_and_gumbel_distributed():
    z = np.zeros(200000, dtype=np.float32)
    k1 = LO.gumbel_keys(z, 7)
    k2 = LO.gumbel_keys(z, 7)
    assert np.array_equal(k1, k2)
    assert abs(k1.mean() - 0.5772156649) < 0.01  # Euler-Mascheroni constant
    assert abs(k1.var() - np.pi ** 2 / 6) < 0.03
    assert not np.array_equal(k1, LO.gumbel_keys(z, 8))


def test_landmark_factor_all_points_is_exact():
    g = np.random.default_rng(3)
    X = g.standard_normal((120, 4))
    y = np.where(g.random(120) < 0.5, 1.0, -1.0)
    Z, nu = LO.landmark_factor(X, y, 0.5, np.arange(120))
    Q = LO.rbf_q(X, X, y, y, 0.5)
    assert np.linalg.norm(Q - Z @ Z.T) <= 1e-4 * np.linalg.norm(Q)
    assert LO.residual_estimate(X, y, 0.5, Z, np.arange(0, 120, 7)) <= 1e-4
