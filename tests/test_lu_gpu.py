"""db200_lu_factorize (GPU LU, FP32) against the LU oracle and the reference's own factors.

Bar:
  * the reference's fixtures (tests/golden/lu_reference.npz, its lu_factorize_partial_pivot<float>): identical
    pivots, factors within 1e-5 of the largest entry (both FP32, different blocking and summation order);
  * the oracle (FP64) on ragged shapes: identical pivots, factors within 1e-4 of the largest entry;
  * large shapes, where FP32 and FP64 rounding may order near-equal pivot candidates differently: the partial
    pivoting properties (|l| <= 1, valid pivot rows) and a backward error ||P A - L U||_F <= 1e-6 n ||A||_F;
  * interchanges reaching the columns left of the block, the replicate-panel variant, no pivoting, a zero pivot.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def gpu_lu(ctx, A, pivot=1, nleft=0, swap_left_panels=1):
    """Factor the block of A (m x (nleft + n), column major) right of its first nleft columns."""
    import torch
    A = np.asfortranarray(A, dtype=np.float32)
    m, cols = A.shape
    n = cols - nleft
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()  # column major bytes
    ip = torch.zeros(max(min(m, n), 1), dtype=torch.int32, device="cuda")
    ctx.lu_factorize(m, n, dA.data_ptr() + 4 * nleft * m, m, ip.data_ptr(), pivot=pivot, nleft=nleft,
                     swap_left_panels=swap_left_panels)
    ctx.sync()
    return np.asfortranarray(dA.cpu().numpy().T), ip.cpu().numpy()[:min(m, n)]


def factors(LU):
    m, n = LU.shape
    mn = min(m, n)
    return np.tril(LU[:, :mn], -1) + np.eye(m, mn), np.triu(LU[:mn, :])


@pytest.mark.parametrize("k", range(4))
def test_lu_matches_reference_fixture(gpu_ctx, k):
    from pathlib import Path
    g = np.load(Path(__file__).resolve().parent / "golden" / "lu_reference.npz")
    A, LU, ipiv = g[f"c{k}_A"], g[f"c{k}_LU"], g[f"c{k}_ipiv"]
    LUg, ipg = gpu_lu(gpu_ctx, A)
    assert np.array_equal(ipg, ipiv)
    assert np.abs(LUg - LU).max() <= 1e-5 * np.abs(LU).max()


@pytest.mark.parametrize("m,n", [(1, 1), (1, 5), (5, 1), (32, 32), (33, 33), (64, 31), (100, 257), (300, 300)])
def test_lu_matches_oracle(gpu_ctx, m, n):
    A = np.random.default_rng(7 * m + n).uniform(-2, 2, (m, n)).astype(np.float32)
    LUo, ipo = O.lu_partial_pivot(A)
    LUg, ipg = gpu_lu(gpu_ctx, A)
    assert np.array_equal(ipg, ipo)
    assert np.abs(LUg - LUo).max() <= 1e-4 * max(1.0, np.abs(LUo).max())


# Trailing matrices of a million entries or more take the tensor-core update (split-fp16 operands, 22 bits,
# fp32 accumulation), the rest the FP32 FMA kernel: both within the same backward-error bound
@pytest.mark.parametrize("m,n", [(2048, 2048), (3000, 1800), (1500, 2600), (4096, 4096)])
def test_lu_large_backward_error(gpu_ctx, m, n):
    A = np.random.default_rng(m + n).uniform(-2, 2, (m, n)).astype(np.float32)
    LUg, ipg = gpu_lu(gpu_ctx, A)
    mn = min(m, n)
    assert np.all(ipg >= np.arange(1, mn + 1)) and np.all(ipg <= m)
    L, U = factors(LUg.astype(np.float64))
    assert np.abs(np.tril(LUg[:, :mn], -1)).max() <= 1.0
    err = np.linalg.norm(L @ U - O.lu_apply_ipiv(A.astype(np.float64), ipg)) / np.linalg.norm(A)
    print(f"LU {m}x{n}: ||PA - LU||_F / ||A||_F = {err:.3e}")
    assert err <= 1e-6 * max(m, n)


def test_lu_interchanges_reach_left_columns(gpu_ctx):
    """lu_factorize_partial_pivot on a block at column j permutes the rows of the columns left of it too."""
    g = np.random.default_rng(11)
    m, left, n = 90, 7, 70
    A = g.uniform(-2, 2, (m, left + n)).astype(np.float32)
    LUg, ipg = gpu_lu(gpu_ctx, A, nleft=left)
    LUo, ipo = O.lu_partial_pivot(A[:, left:])
    assert np.array_equal(ipg, ipo)
    assert np.array_equal(LUg[:, :left], O.lu_apply_ipiv(A[:, :left], ipo))
    assert np.abs(LUg[:, left:] - LUo).max() <= 1e-4 * np.abs(LUo).max()


def test_lu_replicate_panel_keeps_earlier_panels(gpu_ctx):
    """Interchanges reaching only the columns right of each panel: the same pivots and U, L rows unpermuted by later
    panels (so the standard L is the replicate-panel L with each panel's later interchanges applied)."""
    A = np.random.default_rng(12).uniform(-2, 2, (100, 100)).astype(np.float32)
    LUs, ips = gpu_lu(gpu_ctx, A)
    LUr, ipr = gpu_lu(gpu_ctx, A, swap_left_panels=0)
    assert np.array_equal(ips, ipr)
    assert np.array_equal(np.triu(LUs), np.triu(LUr))
    Lr = LUr.copy()
    for k0 in range(0, 100, 32):  # apply each panel's later interchanges to its columns
        cols = slice(k0, min(k0 + 32, 100))
        for j in range(min(k0 + 32, 100), 100):
            p = ipr[j] - 1
            if p != j:
                Lr[[j, p], cols] = Lr[[p, j], cols]
    assert np.array_equal(np.tril(Lr, -1), np.tril(LUs, -1))


def test_lu_no_pivot(gpu_ctx):
    g = np.random.default_rng(3)
    A = (g.uniform(-1, 1, (150, 150)) + 80 * np.eye(150)).astype(np.float32)
    LUo, _ = O.lu_partial_pivot(A, pivot=False)
    LUg, ipg = gpu_lu(gpu_ctx, A, pivot=0)
    assert np.array_equal(ipg, np.arange(1, 151))
    assert np.abs(LUg - LUo).max() <= 1e-5 * np.abs(LUo).max()


def test_lu_zero_pivot_is_reported(gpu_ctx):
    from darray_optimizer_b200._lib import DB200Error
    A = np.random.default_rng(4).uniform(-2, 2, (40, 40)).astype(np.float32)
    A[:, 5] = 0.0  # column 6 has no nonzero entry: a zero pivot at column 6
    with pytest.raises(DB200Error) as e:
        gpu_lu(gpu_ctx, A)
    assert e.value.status == -10 and "column 6" in str(e.value)


def test_grid_barrier_wait_gives_up(gpu_ctx):
    """The LU panel's grid-wide barrier is bounded: with one CTA that never arrives, the others give up after
    20 ms, DB200_ERR_TIMEOUT reaches the host at synchronize, and the context then factors a matrix normally."""
    from darray_optimizer_b200._lib import DB200Error
    assert gpu_ctx.lib.db200_selftest_grid_barrier_timeout(gpu_ctx.h, 20) == 0
    with pytest.raises(DB200Error) as ei:
        gpu_ctx.sync()
    assert ei.value.status == -6  # DB200_ERR_TIMEOUT
    gpu_ctx.sync()  # the status word was cleared
    A = np.random.default_rng(31).uniform(-2, 2, (200, 200)).astype(np.float32)
    LUo, ipo = O.lu_partial_pivot(A)
    LUg, ipg = gpu_lu(gpu_ctx, A)
    assert np.array_equal(ipg, ipo)
    assert np.abs(LUg - LUo).max() <= 1e-4 * np.abs(LUo).max()
