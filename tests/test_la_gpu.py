"""FP64 dense linear algebra on the GPU (through the C ABI) against the FP64 oracle and the reference's own
known answers.  Tolerances: FP64 results agree with numpy/LAPACK to relative 1e-11 (Cholesky, GEMM, TRSM) and
CholeskyQR2 gives Q^T Q = I to 1e-13; against the reference's FP32 outputs (tests/golden) the bar is 1e-4."""
from pathlib import Path

import numpy as np
import pytest

from darray_optimizer_b200._lib import DB200Error
from oracle import oracle as O

pytestmark = pytest.mark.gpu

G = np.load(Path(__file__).resolve().parent / "golden" / "reference_goldens.npz")


def d64(a):
    """column-major FP64 device copy of a 2-D array (torch tensor shaped (cols, rows))."""
    import torch
    a = np.asarray(a, np.float64)
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()


def h64(t, m):
    return np.asfortranarray(t.cpu().numpy()[:, :m].T)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("nb", [64, 32, 17])
def test_potrf_known_answer_min_matrix(gpu_ctx, nb):
    # perftests/perftest_cholesky.cpp:46-84: chol(min(i+1, j+1)) = ones-upper; the reference checks A[n-1,n-1] == 1
    A = G["chol_min_A"].astype(np.float64)
    n = A.shape[0]
    dA = d64(A)
    gpu_ctx.potrf(n, dA.data_ptr(), n, nb)
    R = h64(dA, n)
    assert np.max(np.abs(R - np.triu(np.ones((n, n))))) < 1e-12
    assert abs(R[n - 1, n - 1] - 1.0) < 1e-12
    assert np.max(np.abs(R - G["chol_min_R_blocked"])) < 1e-4  # the reference's own FP32 factor


@pytest.mark.parametrize("n", [10, 200, 528, 1040])
def test_potrf_matches_oracle(gpu_ctx, n):
    g = np.random.default_rng(n)
    B = g.standard_normal((n, n))
    A = B @ B.T / n + np.eye(n)
    dA = d64(A)
    gpu_ctx.potrf(n, dA.data_ptr(), n)
    R = h64(dA, n)
    assert rel(R, O.cholesky_upper(A)) < 1e-11
    assert np.all(np.tril(R, -1) == 0)


@pytest.mark.parametrize("n,nb", [(1, 64), (63, 64), (65, 64), (130, 17), (191, 32), (2064, 64)])
def test_potrf_ragged_blocks(gpu_ctx, n, nb):
    # partial diagonal blocks, partial 64-column panel chunks and block sizes below 64
    g = np.random.default_rng(n + nb)
    B = g.standard_normal((n, n))
    A = B @ B.T / n + 0.5 * np.eye(n)
    dA = d64(A)
    gpu_ctx.potrf(n, dA.data_ptr(), n, nb)
    R = h64(dA, n)
    assert rel(R, O.cholesky_upper(A)) < 1e-11
    assert np.all(np.tril(R, -1) == 0)


@pytest.mark.parametrize("n", [4096, 8192])
def test_potrf_known_answer_large(gpu_ctx, n):
    # perftest_cholesky's sizes: the min(i+1, j+1) matrix of integers factors exactly in FP64 (every pivot 1),
    # so the whole factor must be the upper triangle of ones; the trailing updates run on the DMMA tile path here
    import torch
    i = torch.arange(1, n + 1, device="cuda", dtype=torch.float64)
    A = torch.minimum(i[:, None], i[None, :])
    gpu_ctx.potrf(n, A.data_ptr(), n)
    gpu_ctx.sync()
    # column major upper factor = lower triangle of the row-major view
    assert float((A - torch.tril(torch.ones_like(A))).abs().max()) == 0.0
    assert float(A[n - 1, n - 1]) == 1.0


@pytest.mark.parametrize("n,nb", [(3000, 64), (2500, 48)])
def test_potrf_large_matches_oracle(gpu_ctx, n, nb):
    # both trailing-update paths in one factor: 128 x 128 DMMA tiles while the trailing matrix is large, 32 x 32
    # tiles for the last blocks
    g = np.random.default_rng(n)
    B = g.standard_normal((n, n))
    A = B @ B.T / n + np.eye(n)
    dA = d64(A)
    gpu_ctx.potrf(n, dA.data_ptr(), n, nb)
    R = h64(dA, n)
    assert rel(R, O.cholesky_upper(A)) < 1e-11
    assert np.all(np.tril(R, -1) == 0)


@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 64, 65, 100, 138, 272, 300, 511, 513, 528, 544])
def test_potrf_cluster_matches_oracle(gpu_ctx, n):
    # up to n = 544 the default block size takes the one-launch cluster factor (one kernel, no lower-triangle pass)
    import torch
    g = np.random.default_rng(1000 + n)
    B = g.standard_normal((n, n))
    A = B @ B.T / n + np.eye(n)
    lda = n + 7
    dA = torch.zeros((n, lda), dtype=torch.float64, device="cuda")
    dA[:, :n] = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dA[:, n:] = 5.0  # rows beyond n stay untouched
    low = torch.tril(torch.ones((n, n), dtype=torch.bool, device="cuda"), -1)  # rows i > j of column j
    dA[:, :n][low.T] = float("nan")  # the strictly lower triangle is never read
    l0 = gpu_ctx.launches()
    gpu_ctx.potrf(n, dA.data_ptr(), lda)
    assert gpu_ctx.launches() - l0 == 1
    R = h64(dA, n)
    assert rel(R, O.cholesky_upper(A)) < 1e-11
    assert np.all(np.tril(R, -1) == 0)
    assert bool((dA[:, n:] == 5.0).all())


@pytest.mark.parametrize("n", [96, 528])
def test_potrf_cluster_agrees_with_blocked_path(gpu_ctx, n):
    g = np.random.default_rng(n)
    B = g.standard_normal((n, n))
    A = B @ B.T / n + 0.1 * np.eye(n)
    d1, d2 = d64(A), d64(A)
    gpu_ctx.potrf(n, d1.data_ptr(), n)       # one cluster launch
    gpu_ctx.potrf(n, d2.data_ptr(), n, 32)   # the multi-kernel path
    R1, R2 = h64(d1, n), h64(d2, n)
    assert rel(R1, R2) < 1e-12


@pytest.mark.parametrize("n", [300, 544])
def test_potrf_cluster_known_answer_min_matrix(gpu_ctx, n):
    # min(i+1, j+1) factors exactly (every pivot 1): the factor must be the upper triangle of ones, bit for bit
    import torch
    i = torch.arange(1, n + 1, device="cuda", dtype=torch.float64)
    A = torch.minimum(i[:, None], i[None, :])
    gpu_ctx.potrf(n, A.data_ptr(), n)
    gpu_ctx.sync()
    assert float((A - torch.tril(torch.ones_like(A))).abs().max()) == 0.0


@pytest.mark.parametrize("n,bad", [(300, 0), (300, 31), (300, 32), (300, 150), (300, 299), (544, 520), (5, 4)])
def test_potrf_cluster_not_spd_reports_block(gpu_ctx, n, bad):
    A = np.eye(n)
    A[bad, bad] = -1.0
    dA = d64(A)
    with pytest.raises(DB200Error) as ei:
        gpu_ctx.potrf(n, dA.data_ptr(), n)
    assert ei.value.status == -3  # DB200_ERR_NOT_SPD
    assert f"starting at row {bad // 32 * 32}" in str(ei.value)
    # the context stays usable: an SPD factor right after
    A2 = np.eye(n) * 4.0
    d2 = d64(A2)
    gpu_ctx.potrf(n, d2.data_ptr(), n)
    assert np.allclose(h64(d2, n), 2.0 * np.eye(n))


def test_potrf_cluster_nan_pivot_reports_error(gpu_ctx):
    A = np.eye(200)
    A[77, 77] = np.nan
    dA = d64(A)
    with pytest.raises(DB200Error) as ei:
        gpu_ctx.potrf(200, dA.data_ptr(), 200)
    assert ei.value.status == -3


def test_potrf_test3_factor_and_reference(gpu_ctx):
    A = G["chol_test3_A"].astype(np.float64)
    dA = d64(A)
    gpu_ctx.potrf(10, dA.data_ptr(), 10, 4)
    assert rel(h64(dA, 10), G["chol_test3_R"].astype(np.float64)) < 1e-5


def test_potrf_not_spd_reports_error(gpu_ctx):
    A = np.eye(70)
    A[40, 40] = -1.0
    dA = d64(A)
    with pytest.raises(DB200Error) as ei:
        gpu_ctx.potrf(70, dA.data_ptr(), 70)
    assert ei.value.status == -3  # DB200_ERR_NOT_SPD


@pytest.mark.parametrize("n,l", [(5000, 138), (20000, 528), (500, 20)])
def test_cholqr2_matches_oracle(gpu_ctx, n, l):
    g = np.random.default_rng(l)
    Y = g.standard_normal((n, l)) @ np.diag(np.logspace(0, -4, l))
    dY = d64(Y)
    dR = d64(np.zeros((l, l)))
    gpu_ctx.cholqr2(n, l, dY.data_ptr(), n, dR.data_ptr(), l)
    Q, R = h64(dY, n), h64(dR, l)
    Qo, Ro = O.cholqr2(Y)
    assert np.max(np.abs(Q.T @ Q - np.eye(l))) < 1e-13
    assert rel(Q, Qo) < 1e-10 and rel(R, Ro) < 1e-10
    assert rel(Q @ R, Y) < 1e-13


def test_cholqr2_matches_reference_tsqr(gpu_ctx):
    # tall_skinny_qr_factorize of the reference (FP32 Householder): same Q and R up to signs
    A = G["tsqr_A"].astype(np.float64)
    n, l = A.shape
    dY = d64(A)
    dR = d64(np.zeros((l, l)))
    gpu_ctx.cholqr2(n, l, dY.data_ptr(), n, dR.data_ptr(), l)
    Qr, Rr = O.sign_fix(G["tsqr_Q"].astype(np.float64), G["tsqr_R"].astype(np.float64))
    assert rel(h64(dY, n), Qr) < 1e-5 and rel(h64(dR, l), Rr) < 1e-5


def test_cholqr2_ill_conditioned_uses_shifted_variant(gpu_ctx):
    n, l = 4000, 60
    g = np.random.default_rng(1)
    U, _ = np.linalg.qr(g.standard_normal((n, l)))
    V, _ = np.linalg.qr(g.standard_normal((l, l)))
    Y = U @ np.diag(np.logspace(0, -11, l)) @ V.T  # cond 1e11: the plain Gram is singular in FP64
    dY = d64(Y)
    dR = d64(np.zeros((l, l)))
    gpu_ctx.cholqr2(n, l, dY.data_ptr(), n, dR.data_ptr(), l)
    Q, R = h64(dY, n), h64(dR, l)
    assert np.max(np.abs(Q.T @ Q - np.eye(l))) < 1e-12
    assert rel(Q @ R, Y) < 1e-12
    Qo, Ro = O.cholqr2(Y)
    assert np.max(np.abs(Qo.T @ Qo - np.eye(l))) < 1e-12


def test_gemm_tn_matches_oracle_and_reference(gpu_ctx):
    A, B, C = (G[k].astype(np.float64) for k in ("mm_A", "mm_B", "mm_C"))
    k, m = A.shape
    n = B.shape[1]
    dA, dB, dC = d64(A), d64(B), d64(C)
    gpu_ctx.gemm_tn(k, m, n, -1.0, dA.data_ptr(), k, dB.data_ptr(), k, 1.0, dC.data_ptr(), m)
    gpu_ctx.sync()
    out = h64(dC, m)
    assert rel(out, O.matmul_tn(A, B, C, alpha=-1.0, beta=1.0)) < 1e-13
    assert rel(out, G["mm_out"].astype(np.float64)) < 1e-5


@pytest.mark.parametrize("m,n", [(64, 7), (300, 41)])
def test_trsm_lutn_matches_oracle(gpu_ctx, m, n):
    g = np.random.default_rng(m)
    U = np.triu(g.standard_normal((m, m))) + 8 * np.eye(m)
    B = g.standard_normal((m, n))
    dU, dB = d64(U), d64(B)
    gpu_ctx.trsm_lutn(m, n, dU.data_ptr(), m, dB.data_ptr(), m)
    assert rel(h64(dB, m), O.trsm_lutn(U, B)) < 1e-12
    if m == 64:
        dU2, dB2 = d64(G["trsm_U"]), d64(G["trsm_B"])
        gpu_ctx.trsm_lutn(64, 7, dU2.data_ptr(), 64, dB2.data_ptr(), 64)
        assert rel(h64(dB2, 64), G["trsm_X"].astype(np.float64)) < 1e-5


def test_svd_values_match_reference_and_oracle(gpu_ctx):
    A = G["svd_A"].astype(np.float64)
    n = A.shape[0]
    dA = d64(A)
    import torch
    dS = torch.zeros(n, dtype=torch.float64, device="cuda")
    gpu_ctx.svd_values(n, dA.data_ptr(), n, dS.data_ptr())
    S = dS.cpu().numpy()
    assert rel(S, O.svd_values(A)) < 1e-12
    assert rel(S, G["svd_S"].astype(np.float64)) < 1e-5  # the reference's sgesvd


@pytest.mark.parametrize("ta", ["N", "T"])
def test_sgemm_matches_numpy(gpu_ctx, ta):
    import torch
    g = np.random.default_rng(3)
    m, n, k = 70, 45, 300
    A = g.standard_normal((m, k) if ta == "N" else (k, m)).astype(np.float32)
    B = g.standard_normal((k, n)).astype(np.float32)
    C = g.standard_normal((m, n)).astype(np.float32)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    dC = torch.from_numpy(np.ascontiguousarray(C.T)).cuda()
    lda = A.shape[0]
    gpu_ctx.sgemm(ta, "N", m, n, k, 1.5, dA.data_ptr(), lda, dB.data_ptr(), k, -0.5, dC.data_ptr(), m)
    gpu_ctx.sync()
    opA = A.astype(np.float64) if ta == "N" else A.astype(np.float64).T
    ref = 1.5 * opA @ B - 0.5 * C
    assert rel(dC.cpu().numpy().T, ref) < 1e-6


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N")])
def test_gemm_matches_numpy(gpu_ctx, ta, tb):
    g = np.random.default_rng(4)
    m, n, k = 90, 33, 200
    A = g.standard_normal((m, k) if ta == "N" else (k, m))
    B = g.standard_normal((k, n) if tb == "N" else (n, k))
    C = g.standard_normal((m, n))
    dA, dB, dC = d64(A), d64(B), d64(C)
    gpu_ctx.gemm(ta, tb, m, n, k, 2.0, dA.data_ptr(), A.shape[0], dB.data_ptr(), B.shape[0], 0.25, dC.data_ptr(), m)
    gpu_ctx.sync()
    opA = A if ta == "N" else A.T
    opB = B if tb == "N" else B.T
    assert rel(h64(dC, m), 2.0 * opA @ opB + 0.25 * C) < 1e-13


@pytest.mark.parametrize("n,r,tc", [(2048, 56, 1), (5000, 300, 1), (131, 70, 1), (5000, 300, 0)])
def test_gram_weighted_matches_numpy(gpu_ctx, n, r, tc):
    """Capacity-matrix SYRK Z^T diag(w) Z: FP64 pipes to 1e-13, int8 tensor cores (7 Ozaki slices) to 1e-11
    (upper triangle)."""
    import torch
    g = np.random.default_rng(n + r)
    Z = g.standard_normal((n, r)) * 0.3
    w = np.exp(g.uniform(-6, 6, n))
    dZ = d64(Z)
    dw = torch.from_numpy(w).cuda()
    dM = d64(np.full((r, r), 7.0))
    gpu_ctx.gram_weighted(n, r, dZ.data_ptr(), n, dw.data_ptr(), dM.data_ptr(), r, tc)
    gpu_ctx.sync()
    M = np.triu(h64(dM, r))
    ref = np.triu(Z.T @ (w[:, None] * Z))
    assert rel(M, ref) < (1e-11 if tc else 1e-13)


@pytest.mark.parametrize("n,r,spread", [(3000, 56, 6.0), (1500, 150, 30.0), (131, 70, 6.0), (4096, 200, 2.0),
                                         (40000, 40, 10.0)])
def test_gram_int8_matches_sliced_oracle(gpu_ctx, n, r, spread):
    """The int8 tensor-core Gram equals the exact-integer CPU restatement of the same slicing up to FP64 rounding
    of the final scaling and the split-k atomic additions, including a zero column and zero weights, with weights
    spanning up to 1e26 (the barrier's D^-1 late in a solve)."""
    import torch
    from oracle import ozaki
    g = np.random.default_rng(n + r + int(spread))
    Z = g.standard_normal((n, r)) * np.exp(g.uniform(-3, 3, r))[None, :]
    Z[:, r // 3] = 0.0
    w = np.exp(g.uniform(-spread, spread, n))
    w[::17] = 0.0
    dZ, dw = d64(Z), torch.from_numpy(w).cuda()
    dM = d64(np.zeros((r, r)))
    gpu_ctx.gram_weighted(n, r, dZ.data_ptr(), n, dw.data_ptr(), dM.data_ptr(), r, 1)
    gpu_ctx.sync()
    M = h64(dM, r)
    S = ozaki.sliced_gram(Z, w, 8)
    exact = Z.T @ (w[:, None] * Z)
    d = np.sqrt(np.diag(exact))
    scale = np.outer(d, d) + 1e-300
    iu = np.triu_indices(r)
    assert np.max(np.abs(M - S)[iu] / scale[iu]) < 1e-14
    assert np.max(np.abs(M - exact)[iu] / scale[iu]) < 1e-11
    assert np.all(np.tril(M, -1) == 0)


@pytest.mark.parametrize("slices,bound", [(5, 1e-7), (6, 2e-9), (7, 2e-11)])
def test_gram_int8_fewer_slices_match_sliced_oracle(gpu_ctx, slices, bound):
    """The int8 Gram with 5..7 digits per value (fewer tensor-core products, the barrier's first capacity
    matrices) equals the exact-integer restatement of the same slicing, and stays within the slicing's error of the
    exact Gram."""
    import torch
    from oracle import ozaki
    n, r = 20000, 96
    g = np.random.default_rng(slices)
    Z = g.standard_normal((n, r)) * np.exp(g.uniform(-3, 3, r))[None, :]
    w = np.exp(g.uniform(-8, 8, n))
    dZ, dw = d64(Z), torch.from_numpy(w).cuda()
    dM = d64(np.zeros((r, r)))
    gpu_ctx.gram_weighted(n, r, dZ.data_ptr(), n, dw.data_ptr(), dM.data_ptr(), r, slices)
    gpu_ctx.sync()
    M = h64(dM, r)
    S = ozaki.sliced_gram(Z, w, slices)
    exact = Z.T @ (w[:, None] * Z)
    d = np.sqrt(np.diag(exact))
    scale = np.outer(d, d) + 1e-300
    iu = np.triu_indices(r)
    assert np.max(np.abs(M - S)[iu] / scale[iu]) < 1e-14
    assert np.max(np.abs(M - exact)[iu] / scale[iu]) < bound
