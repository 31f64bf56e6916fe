"""The integer-sliced Gram restatement (oracle/ozaki.py) that pins the GPU's int8 tensor-core capacity matrix:
its digits reconstruct every scaled value to 2^-49 of its column maximum, and its Gram agrees with the exact FP64
Z^T diag(w) Z to 1e-11 of the Cauchy-Schwarz bound ||z_p|| ||z_q|| for 7 slices (and improves ~100x per slice)."""
import numpy as np
import pytest

from oracle import ozaki


def test_digits_reconstruct_and_stay_in_int8_range():
    g = np.random.default_rng(1)
    Zw = g.standard_normal((500, 9)) * np.exp(g.uniform(-20, 20, 9))[None, :]
    Zw[:, 4] = 0.0
    e = ozaki.col_exponents(Zw)
    assert np.all(np.max(np.abs(Zw), axis=0) < np.ldexp(1.0, e))
    D = ozaki.digits(Zw, e, 7)
    assert D.min() >= -127 and D.max() <= 127
    back = sum(np.ldexp(D[s].astype(float), e[None, :] - 7 * (s + 1)) for s in range(7))
    colmax = np.max(np.abs(Zw), axis=0)
    assert np.all(np.abs(back - Zw) <= np.ldexp(1.0, e - 49)[None, :])
    assert np.all(np.abs(back - Zw)[:, colmax > 0] <= 2.0 ** -48 * colmax[colmax > 0][None, :])


@pytest.mark.parametrize("ks,bound", [(5, 2e-8), (6, 3e-10), (7, 3e-12), (8, 3e-14)])
def test_sliced_gram_error_per_slice_count(ks, bound):
    g = np.random.default_rng(ks)
    n, r = 3000, 40
    Z = g.standard_normal((n, r)) * 0.3
    w = np.exp(g.uniform(-20, 20, n))
    exact = Z.T @ (w[:, None] * Z)
    d = np.sqrt(np.diag(exact))
    err = np.max(np.abs(ozaki.sliced_gram(Z, w, ks) - exact) / np.outer(d, d))
    assert err < bound


def test_chunked_scaling_matches_exact_gram_across_chunks():
    # 16384-row chunks carry their own column exponents; a column whose size changes by 1e8 between chunks keeps
    # full relative accuracy in both
    g = np.random.default_rng(7)
    n, r = 40000, 12
    Z = g.standard_normal((n, r))
    Z[:16384, 3] *= 1e-8
    w = np.exp(g.uniform(-5, 5, n))
    exact = Z.T @ (w[:, None] * Z)
    d = np.sqrt(np.diag(exact))
    assert np.max(np.abs(ozaki.sliced_gram(Z, w, 7) - exact) / np.outer(d, d)) < 3e-12
    part = Z[:16384].T @ (w[:16384, None] * Z[:16384])
    dp = np.sqrt(np.diag(part))
    assert np.max(np.abs(ozaki.sliced_gram(Z[:16384], w[:16384], 7) - part) / np.outer(dp, dp)) < 3e-12
