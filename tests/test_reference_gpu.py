"""The reference's own GPU kernel-block code (include/dkernel.cu: rbf_kernel, tc_gemm; compiled unmodified for
sm_100a into oracle/_ref/libdkernel_ref.so by oracle/build_ref.sh) run on the same host inputs as the FP64
oracle and as the product library's drop-in symbols of the same names.

This pins the oracle's kernel-block and sketch restatements against the reference itself, and shows that the
drop-in entry points give the reference's results.

Tolerances:
  * reference rbf_kernel vs oracle.rbf_block: max |dK| <= 1e-5.  The reference forms distances with a cuBLAS
    FP32 GEMM and applies __expf.
  * reference LRA block (rbf_kernel then tc_gemm) vs oracle.sketch: relative Frobenius error <= 1e-5.
  * drop-in rbf_kernel vs reference: max |dK| <= 2e-5 (split-bf16 distance products).
  * drop-in tc_gemm vs reference: relative Frobenius error <= 1e-5 (FP32 data; FP64 against FP32 accumulation).
  * device sketch db200_rbf_sketch vs the reference LRA block: relative Frobenius error <= 2e-3 (fp16 kernel
    tile and sketch operands, fp32 accumulation).

tc_gemm passes beta = 0 to every 8192-column block (include/dkernel.cu:204-218), so for n > 8192 only the last
block's product survives; the cases here keep n <= 8192.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from util import colmajor_empty, colmajor_host, dev, ptr, rel_fro

pytestmark = pytest.mark.gpu

_fp = ctypes.POINTER(ctypes.c_float)
_i, _f = ctypes.c_int, ctypes.c_float


def _p(a):
    return a.ctypes.data_as(_fp)


@pytest.fixture(scope="module")
def ref():
    from pathlib import Path
    lib_path = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libdkernel_ref.so"
    if not lib_path.exists():
        pytest.skip("oracle/_ref/libdkernel_ref.so is not built (oracle/build_ref.sh needs the reference sources)")
    lib = ctypes.CDLL(str(lib_path))
    lib.ref_cuda_init.argtypes = []
    lib.ref_rbf_kernel.argtypes = [_i, _i, _i, _fp, _fp, _fp, _fp, _fp, _i, _f]
    lib.ref_tc_gemm.argtypes = [_i, _i, _i, _fp, _i, _fp, _i, _fp, _i, _f]
    lib.ref_cuda_init()
    return lib


@pytest.fixture(scope="module")
def dropin(gpu_ctx):
    lib = gpu_ctx.lib
    rbf = getattr(lib, "_Z10rbf_kerneliiiiPfiS_iS_S_S_if")
    rbf.argtypes = [_i, _i, _i, _i, _fp, _i, _fp, _i, _fp, _fp, _fp, _i, _f]
    rbf.restype = None
    gemm = getattr(lib, "_Z7tc_gemmiiiiPfiS_iS_iff")
    gemm.argtypes = [_i, _i, _i, _i, _fp, _i, _fp, _i, _fp, _i, _f, _f]
    gemm.restype = None
    getattr(lib, "_Z9cuda_initv")()
    return rbf, gemm


def _points(n, d, seed):
    g = np.random.default_rng(seed)
    return g.standard_normal((n, d)).astype(np.float32)


def _labels(n, seed):
    g = np.random.default_rng(seed + 7)
    return np.where(g.random(n) < 0.5, 1.0, -1.0).astype(np.float32)


def ref_rbf(lib, Xi, Xj, yi, yj, gamma):
    m, d = Xi.shape
    n = Xj.shape[0]
    xi, xj = np.asfortranarray(Xi), np.asfortranarray(Xj)
    K = np.zeros((m, n), np.float32, order="F")
    lib.ref_rbf_kernel(m, n, d, _p(xi), _p(xj), _p(yi), _p(yj), _p(K), m, float(gamma))
    return K


def ref_gemm(lib, A, Bm):
    m, n = A.shape
    k = Bm.shape[1]
    a, b = np.asfortranarray(A), np.asfortranarray(Bm)
    C = np.zeros((m, k), np.float32, order="F")
    lib.ref_tc_gemm(m, k, n, _p(a), m, _p(b), n, _p(C), m, 1.0)
    return C


@pytest.mark.parametrize("m,n,d", [(300, 257, 20), (1, 5, 3), (77, 390, 64), (1024, 700, 128)])
def test_reference_rbf_kernel_pins_oracle_and_dropin(ref, dropin, m, n, d):
    Xi, Xj = _points(m, d, 11), _points(n, d, 12)
    yi, yj = _labels(m, 11), _labels(n, 12)
    gamma = np.float32(0.7 / d)
    Kr = ref_rbf(ref, Xi, Xj, yi, yj, gamma)
    assert np.max(np.abs(Kr - O.rbf_block(Xi, Xj, yi, yj, float(gamma)))) <= 1e-5
    # drop-in symbol, same host buffers, leading dimension of K larger than m
    rbf, _ = dropin
    ldk = m + 5
    Kd = np.zeros((ldk, n), np.float32, order="F")
    xi, xj = np.asfortranarray(Xi), np.asfortranarray(Xj)
    rbf(0, m, n, d, _p(xi), m, _p(xj), n, _p(yi), _p(yj), _p(Kd), ldk, gamma)
    assert np.max(np.abs(Kd[:m] - Kr)) <= 2e-5


@pytest.mark.parametrize("n,d,l", [(2048, 32, 70), (1000, 17, 33), (300, 8, 5)])
def test_reference_lra_block_pins_sketch(ref, dropin, gpu_ctx, n, d, l):
    g = np.random.default_rng(n + d + l)
    y = np.where(g.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    X = (g.standard_normal((n, d)) + 0.5 * y[:, None]).astype(np.float32)
    Om = g.standard_normal((n, l)).astype(np.float32)
    gamma = np.float32(1.0 / d)
    Kr = ref_rbf(ref, X, X, y, y, gamma)
    Yr = ref_gemm(ref, Kr, Om)
    assert rel_fro(Yr, O.sketch(X, X, y, y, Om, float(gamma))) <= 1e-5
    # drop-in tc_gemm on the reference's K
    _, gemm = dropin
    Yd = np.zeros((n, l), np.float32, order="F")
    kr, om = np.asfortranarray(Kr), np.asfortranarray(Om)
    gemm(0, n, l, n, _p(kr), n, _p(om), n, _p(Yd), n, 1.0, 0.0)
    assert rel_fro(Yd, Yr) <= 1e-5
    # the device-resident fused sketch (K never stored) against the reference's two-step block
    dX, dy, dO = dev(X), dev(y), dev(np.asfortranarray(Om))
    Y = colmajor_empty(n, l)
    gpu_ctx.rbf_sketch(n, n, d, l, ptr(dX), d, ptr(dX), d, 0, ptr(dy), ptr(dy), ptr(dO), n, ptr(Y), n,
                       float(gamma))
    gpu_ctx.sync()
    assert rel_fro(colmajor_host(Y, n), Yr) <= 2e-3


def test_reference_tc_gemm_single_block_paths(ref, dropin):
    """jb >= 256 takes cublasGemmEx, jb < 256 cublasSgemm (include/dkernel.cu:204-218); both against the
    drop-in tc_gemm and an FP64 product."""
    _, gemm = dropin
    g = np.random.default_rng(5)
    for m, k, n in [(640, 48, 1000), (129, 7, 200)]:
        A = g.standard_normal((m, n)).astype(np.float32)
        Bm = g.standard_normal((n, k)).astype(np.float32)
        Cr = ref_gemm(ref, A, Bm)
        exact = A.astype(np.float64) @ Bm.astype(np.float64)
        assert rel_fro(Cr, exact) <= 1e-5
        Cd = np.zeros((m, k), np.float32, order="F")
        a, b = np.asfortranarray(A), np.asfortranarray(Bm)
        gemm(0, m, k, n, _p(a), m, _p(b), n, _p(Cd), m, 1.0, 0.0)
        assert rel_fro(Cd, Cr) <= 1e-5
