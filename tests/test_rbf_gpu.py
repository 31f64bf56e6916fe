"""Parity of the tcgen05 RBF tile engine (through the C ABI) against the FP64 oracle.

Tolerances (stated here, checked below):
  * db200_rbf_block: |K_gpu - K_oracle| <= 2e-5 elementwise.  Distances come from split-fp16 products of points
    scaled by a power of two (22 significant bits per coordinate), exp2 and norms in fp32.
  * db200_rbf_sketch: ||Y_gpu - Y_oracle||_F <= 2e-3 ||Y_oracle||_F.  The kernel tile P and Omega enter the
    sketch product as fp16 (relative rounding 2^-12 each) with fp32 accumulation (measured ~3e-4).
  * db200_rbf_sketch_ex: compensated product (P and Omega each as fp16 hi + lo) <= 6e-5 relative Frobenius (the
    tensor cores' truncating fp32 accumulation over n points); with the accumulation promoted every 256 points
    <= 3e-6; P split only <= 4e-4.
  * at the full C2 size (n = 131072, d = 128, l = 528) on 64 sampled rows against the FP64 oracle: the single
    product <= 6e-4 (measured 3.0e-4), the promoted compensated product <= 3e-6 (measured 1.3e-6).
"""
import numpy as np
import pytest

from oracle import oracle as O
from util import colmajor_empty, colmajor_host, dev, ptr, rel_fro

pytestmark = pytest.mark.gpu

POINT_MAJOR, FEATURE_MAJOR = 0, 1


def _points(n, d, seed, scale=1.0):
    g = np.random.default_rng(seed)
    return (scale * g.standard_normal((n, d))).astype(np.float32)


def _labels(n, seed):
    g = np.random.default_rng(seed + 100)
    return np.where(g.random(n) < 0.5, 1.0, -1.0).astype(np.float32)


@pytest.mark.parametrize("m,n,d,layout", [
    (128, 128, 32, POINT_MAJOR),
    (300, 257, 20, POINT_MAJOR),
    (1000, 1000, 128, POINT_MAJOR),
    (77, 390, 64, FEATURE_MAJOR),
    (1, 5, 3, POINT_MAJOR),
])
def test_rbf_block_matches_oracle(gpu_ctx, m, n, d, layout):
    Xi, Xj = _points(m, d, 1), _points(n, d, 2)
    yi, yj = _labels(m, 1), _labels(n, 2)
    gamma = 0.7 / d
    Kref = O.rbf_block(Xi, Xj, yi, yj, gamma)
    if layout == POINT_MAJOR:
        dXi, dXj, ldxi, ldxj = dev(Xi), dev(Xj), d, d
    else:  # m x d column major: store X^T row-major
        dXi, dXj, ldxi, ldxj = dev(np.asfortranarray(Xi)), dev(np.asfortranarray(Xj)), m, n
    ldk = m + 3
    K = colmajor_empty(m, n, ldk)
    dyi, dyj = dev(yi), dev(yj)  # keep the device buffers alive across the call
    gpu_ctx.rbf_block(m, n, d, ptr(dXi), ldxi, ptr(dXj), ldxj, layout, ptr(dyi), ptr(dyj), ptr(K), ldk, gamma)
    gpu_ctx.sync()
    Kg = colmajor_host(K, m)
    assert np.max(np.abs(Kg - Kref)) <= 2e-5


def test_rbf_block_symmetric_unit_diagonal(gpu_ctx):
    n, d = 512, 48
    X = _points(n, d, 5, scale=0.3)
    dX = dev(X)
    K = colmajor_empty(n, n)
    gpu_ctx.rbf_block(n, n, d, ptr(dX), d, ptr(dX), d, POINT_MAJOR, 0, 0, ptr(K), n, 1.0 / d)
    gpu_ctx.sync()
    Kg = colmajor_host(K, n)
    assert np.allclose(np.diag(Kg), 1.0, atol=1e-5)
    assert np.max(np.abs(Kg - Kg.T)) <= 1e-5
    assert Kg.min() > 0 and Kg.max() <= 1.0 + 1e-6


@pytest.mark.parametrize("m,n,d,l", [
    (256, 256, 32, 16),
    (1000, 1000, 20, 40),
    (300, 777, 128, 200),
    (512, 512, 64, 528),
    (130, 4096, 32, 138),
    # wider than one tile-kernel panel: the cluster kernel, 1, 2 and 4 super-panels, ragged m, n and d
    (700, 900, 100, 600),
    (300, 257, 7, 1040),
    (1024, 2048, 128, 2064),
])
def test_rbf_sketch_matches_oracle(gpu_ctx, m, n, d, l):
    Xi = _points(m, d, 11, 0.5)
    Xj = Xi if m == n else _points(n, d, 12, 0.5)
    yi = _labels(m, 3)
    yj = yi if m == n else _labels(n, 4)
    g = np.random.default_rng(9)
    Om = np.asfortranarray(g.standard_normal((n, l)).astype(np.float32))
    gamma = 1.0 / d
    Yref = O.sketch(Xi, Xj, yi, yj, Om, gamma)
    dXi = dev(Xi)
    dXj = dXi if Xj is Xi else dev(Xj)
    dyi = dev(yi)
    dyj = dyi if yj is yi else dev(yj)
    ldy = m + 1
    Y = colmajor_empty(m, l, ldy)
    dOm = dev(Om)
    gpu_ctx.rbf_sketch(m, n, d, l, ptr(dXi), d, ptr(dXj), d, POINT_MAJOR, ptr(dyi), ptr(dyj), ptr(dOm), n, ptr(Y),
                       ldy, gamma)
    gpu_ctx.sync()
    Yg = colmajor_host(Y, m)
    # fp16 P and Omega~ in the sketch product: ~3e-4 relative in Frobenius norm
    err = rel_fro(Yg, Yref)
    assert err <= 2e-3, err
    # every column against the RMS column norm, so a dropped panel cannot hide behind the global norm
    # (single columns can nearly cancel when K has a dominant constant mode, so not per-column relative)
    rms_col = np.linalg.norm(Yref) / np.sqrt(l)
    col = (np.linalg.norm(Yg - Yref, axis=0) / rms_col).max()
    assert col <= 6e-3, col


@pytest.mark.parametrize("m,n,d,l,seed", [
    (256, 256, 32, 16, 1),
    (1000, 1000, 20, 40, 2),
    (300, 777, 128, 200, 3),
    (512, 512, 64, 528, 4),     # three compensated panels
    (4096, 4096, 32, 138, 5),   # the two-Gaussian workload's sketch width
    (700, 900, 100, 600, 6),
    (300, 257, 7, 1040, 7),
])
def test_rbf_sketch_compensated_matches_oracle(gpu_ctx, m, n, d, l, seed):
    """The compensated sketch product (fp16 hi + lo for both P and Omega) against the FP64 oracle: 22-bit
    operands, so the error falls from ~3e-4 (single product) to the fp32 accumulation and exp2 level."""
    from darray_optimizer_b200 import _lib
    Xi = _points(m, d, 20 + seed, 0.5)
    Xj = Xi if m == n else _points(n, d, 40 + seed, 0.5)
    yi = _labels(m, 5 + seed)
    yj = yi if m == n else _labels(n, 60 + seed)
    g = np.random.default_rng(70 + seed)
    Om = np.asfortranarray(g.standard_normal((n, l)).astype(np.float32))
    gamma = 1.0 / d
    Yref = O.sketch(Xi, Xj, yi, yj, Om, gamma)
    dXi = dev(Xi)
    dXj = dXi if Xj is Xi else dev(Xj)
    dyi = dev(yi)
    dyj = dyi if yj is yi else dev(yj)
    dOm = dev(Om)
    errs = {}
    # compensated: the truncating fp32 accumulation of the tensor cores shrinks long sums by ~2^-25 per step
    # (measured 1.4e-5 at n = 4096); promoted every 256 points it stays at one chunk's worth
    for product, tol in ((_lib.SKETCH_COMPENSATED_PROMOTED, 3e-6), (_lib.SKETCH_COMPENSATED, 6e-5),
                         (_lib.SKETCH_P_SPLIT, 4e-4)):
        Y = colmajor_empty(m, l, m + 1)
        gpu_ctx.rbf_sketch_ex(m, n, d, l, ptr(dXi), d, ptr(dXj), d, POINT_MAJOR, ptr(dyi), ptr(dyj), ptr(dOm), n,
                              ptr(Y), m + 1, gamma, product)
        gpu_ctx.sync()
        errs[product] = rel_fro(colmajor_host(Y, m), Yref)
        assert errs[product] <= tol, (product, errs)


@pytest.mark.parametrize("perturb", [False, True])
def test_rbf_sketch_binary_features(gpu_ctx, perturb):
    """Sparse binary features (x in {0, 1}, Bernoulli(0.11), d = 123, the sparse-binary workload's shape): every
    point is exact in fp16, so the distance products reduce to hi.hi.  With one perturbed coordinate the set is no
    longer exact and the full split runs.  Both against the FP64 oracle, single and compensated products."""
    from darray_optimizer_b200 import _lib
    n, d, l = 2048, 123, 264
    g = np.random.default_rng(31)
    X = (g.random((n, d)) < 0.11).astype(np.float32)
    if perturb:
        X[17, 5] = 0.3
    y = _labels(n, 9)
    Om = np.asfortranarray(g.standard_normal((n, l)).astype(np.float32))
    gamma = 0.05
    Yref = O.sketch(X, X, y, y, Om, gamma)
    dX, dy, dOm = dev(X), dev(y), dev(Om)
    for product, tol in ((_lib.SKETCH_SINGLE, 2e-3), (_lib.SKETCH_COMPENSATED_PROMOTED, 3e-6)):
        Y = colmajor_empty(n, l)
        gpu_ctx.rbf_sketch_ex(n, n, d, l, ptr(dX), d, ptr(dX), d, POINT_MAJOR, ptr(dy), ptr(dy), ptr(dOm), n, ptr(Y),
                              n, gamma, product)
        gpu_ctx.sync()
        err = rel_fro(colmajor_host(Y, n), Yref)
        assert err <= tol, (product, perturb, err)


def test_rbf_sketch_two_calls_reuse_workspace(gpu_ctx):
    n, d, l = 640, 16, 24
    X = _points(n, d, 21)
    y = _labels(n, 21)
    Om = np.asfortranarray(np.random.default_rng(3).standard_normal((n, l)).astype(np.float32))
    dX, dy, dO = dev(X), dev(y), dev(Om)
    outs = []
    for _ in range(2):
        Y = colmajor_empty(n, l)
        gpu_ctx.rbf_sketch(n, n, d, l, ptr(dX), d, ptr(dX), d, POINT_MAJOR, ptr(dy), ptr(dy), ptr(dO), n, ptr(Y), n,
                           0.1)
        gpu_ctx.sync()
        outs.append(colmajor_host(Y, n))
    assert np.array_equal(outs[0], outs[1])  # deterministic: same tiles, same order


@pytest.mark.parametrize("m,n,d,l", [
    (300, 777, 33, 40),      # ragged rows, points and features; one 144-column tile
    (1000, 1000, 128, 138),  # the two-Gaussian workload's width
    (1, 5, 3, 1),            # one row, one column (16-column tile), n not a multiple of 8
    (129, 64, 8, 16),
    (200, 301, 100, 528),    # two 264-column tiles
    (64, 1000, 256, 300),    # widest features; 300 = 264 + 36
    (513, 257, 17, 1040),    # four tiles
])
def test_rbf_sketch_f64_matches_oracle(gpu_ctx, m, n, d, l):
    """The plain FP64 comparator pass (one fused launch on the FP64 tensor cores) agrees with the FP64 oracle to
    relative 1e-12, and every column to 1e-11 of the RMS column norm."""
    import torch
    Xi = _points(m, d, 31, 0.5)
    Xj = Xi if m == n else _points(n, d, 32, 0.5)
    yi, yj = _labels(m, 5), _labels(n, 6)
    Om = np.asfortranarray(np.random.default_rng(2).standard_normal((n, l)))
    gamma = 1.0 / d
    Yref = O.sketch(Xi, Xj, yi, yj, Om, gamma)
    dXi, dXj, dyi, dyj = dev(Xi), dev(Xj), dev(yi), dev(yj)
    dOm = torch.from_numpy(np.ascontiguousarray(Om.T)).cuda()
    Y = torch.zeros((l, m), dtype=torch.float64, device="cuda")
    gpu_ctx.rbf_sketch_f64(m, n, d, l, ptr(dXi), d, ptr(dXj), d, ptr(dyi), ptr(dyj), ptr(dOm), n, ptr(Y), m, gamma)
    gpu_ctx.sync()
    Yg = Y.cpu().numpy().T
    assert rel_fro(Yg, Yref) <= 1e-12
    rms_col = np.linalg.norm(Yref) / np.sqrt(l)
    assert (np.linalg.norm(Yg - Yref, axis=0) / rms_col).max() <= 1e-11


@pytest.mark.parametrize("m,n,d", [(300, 777, 33), (1, 5, 3), (1024, 129, 128)])
def test_rbf_block_f64_matches_oracle(gpu_ctx, m, n, d):
    """The materialised FP64 block: relative 1e-13 elementwise against the oracle."""
    import torch
    Xi, Xj = _points(m, d, 41, 0.5), _points(n, d, 42, 0.5)
    yi, yj = _labels(m, 7), _labels(n, 8)
    gamma = 0.9 / d
    Kref = O.rbf_block(Xi, Xj, yi, yj, gamma)
    dXi, dXj, dyi, dyj = dev(Xi), dev(Xj), dev(yi), dev(yj)
    K = torch.zeros((n, m + 2), dtype=torch.float64, device="cuda")
    gpu_ctx.rbf_block_f64(m, n, d, ptr(dXi), d, ptr(dXj), d, ptr(dyi), ptr(dyj), ptr(K), m + 2, gamma)
    gpu_ctx.sync()
    Kg = K.cpu().numpy()[:, :m].T
    assert np.max(np.abs(Kg - Kref)) <= 1e-13


def test_bounded_wait_expiry_reports_timeout_and_context_survives(gpu_ctx):
    """A device wait on a flag nothing sets runs out after 20 ms: DB200_ERR_TIMEOUT at synchronize, then the same
    context runs a sketch normally."""
    from darray_optimizer_b200._lib import DB200Error
    assert gpu_ctx.lib.db200_selftest_wait_timeout(gpu_ctx.h, 20) == 0
    with pytest.raises(DB200Error) as ei:
        gpu_ctx.sync()
    assert ei.value.status == -6  # DB200_ERR_TIMEOUT
    gpu_ctx.sync()  # the status word was cleared
    n, d, l = 256, 16, 16
    X = _points(n, d, 3)
    y = _labels(n, 3)
    Om = np.asfortranarray(np.random.default_rng(1).standard_normal((n, l)).astype(np.float32))
    dX, dy, dO = dev(X), dev(y), dev(Om)
    Y = colmajor_empty(n, l)
    gpu_ctx.rbf_sketch(n, n, d, l, ptr(dX), d, ptr(dX), d, POINT_MAJOR, ptr(dy), ptr(dy), ptr(dO), n, ptr(Y), n, 0.1)
    gpu_ctx.sync()
    err = rel_fro(colmajor_host(Y, n), O.sketch(X, X, y, y, Om, 0.1))
    assert err <= 2e-3, err


@pytest.mark.parametrize("pinned,pad", [(False, 0), (True, 0), (True, 5)])
def test_lra_host_matches_oracle(gpu_ctx, pinned, pad):
    """db200_lra_host (DArray::LRA's host-pointer convention): pageable result buffers take the staged copy,
    page-locked ones are written by the kernel directly; both give the oracle's sketch (fp16 sketch operands:
    relative Frobenius error <= 2e-3), and rows past n of a padded result stay untouched."""
    import torch
    n, d, k = 1000, 24, 40
    X = _points(n, d, 21, 0.5)
    y = _labels(n, 21)
    g = np.random.default_rng(22)
    Om = np.asfortranarray(g.standard_normal((n, k)).astype(np.float32))
    gamma = 1.0 / d
    ref = O.sketch(X, X, y, y, Om, gamma)
    lda = n + pad
    Xh = torch.from_numpy(np.ascontiguousarray(X))
    yh = torch.from_numpy(y)
    Oh = torch.from_numpy(np.ascontiguousarray(Om.T))
    Ah = torch.full((k, lda), 7.0, dtype=torch.float32)
    if pinned:
        Xh, yh, Oh, Ah = Xh.pin_memory(), yh.pin_memory(), Oh.pin_memory(), Ah.pin_memory()
    gpu_ctx.lra_host(n, d, k, Xh.data_ptr(), d, yh.data_ptr(), Oh.data_ptr(), n, Ah.data_ptr(), lda, gamma)
    A = Ah.numpy()
    assert rel_fro(A[:, :n].T, ref) <= 2e-3
    assert np.all(A[:, n:] == 7.0)


@pytest.mark.parametrize("product,tol", [(0, 6e-4), (3, 3e-6)])  # DB200_SKETCH_SINGLE, _COMPENSATED_PROMOTED
def test_rbf_sketch_full_size_sampled_rows(gpu_ctx, product, tol):
    """The C2 workload at full size (n = 131072, d = 128, l = 528, gamma = 0.5/d, uniform [0,1)^128 points with
    hyperplane labels): the GPU pass over all rows, 64 seeded rows of it against the FP64 oracle's rows."""
    import torch
    from darray_optimizer_b200 import datagen
    w = datagen.uniform_hyperplane()
    Om = w.omega()
    n, d, l = w.n, w.d, w.l
    assert (n, d, l) == (131072, 128, 528)
    dX, dy, dO = dev(w.X), dev(w.y), dev(Om)
    Y = torch.zeros((l, n), dtype=torch.float32, device="cuda")
    gpu_ctx.rbf_sketch_ex(n, n, d, l, ptr(dX), d, ptr(dX), d, POINT_MAJOR, ptr(dy), ptr(dy), ptr(dO), n, ptr(Y), n,
                          w.gamma, product)
    gpu_ctx.sync()
    rows = np.sort(np.random.default_rng(64).choice(n, 64, replace=False))
    Yg = Y[:, torch.from_numpy(rows).cuda()].cpu().numpy().T  # 64 x l
    ref = O.sketch(w.X[rows], w.X, w.y[rows], w.y, Om, w.gamma)
    err = rel_fro(Yg, ref)
    print(f"C2 full size, product {product}: sampled-row error vs FP64 {err:.3e}")
    assert err <= tol
