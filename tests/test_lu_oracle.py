"""The LU oracle (oracle.lu_partial_pivot) against the reference's own lu_factorize_partial_pivot<float>
(include/lapack_like.h:179-279, compiled from its sources at one rank into oracle/_ref): the committed fixture
tests/golden/lu_reference.npz (tests/golden/gen_lu_goldens.py) and, when the library is built, live runs.

Bar: identical pivots; factors within 2e-5 of the largest entry (the reference computes in FP32, the oracle in
FP64); P A = L U for the oracle to FP64 round-off.
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

GOLD = Path(__file__).resolve().parent / "golden" / "lu_reference.npz"
REF_LIB = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libdarray_ref.so"


def factors(LU):
    m, n = LU.shape
    mn = min(m, n)
    L = np.tril(LU[:, :mn], -1) + np.eye(m, mn)
    U = np.triu(LU[:mn, :])
    return L, U


@pytest.mark.parametrize("k", range(4))
def test_oracle_matches_reference_fixture(k):
    g = np.load(GOLD)
    A, LU, ipiv = g[f"c{k}_A"], g[f"c{k}_LU"], g[f"c{k}_ipiv"]
    LUo, ipo = O.lu_partial_pivot(A)
    assert np.array_equal(ipo, ipiv)
    assert np.abs(LUo - LU).max() <= 2e-5 * np.abs(LUo).max()


@pytest.mark.parametrize("m,n", [(1, 1), (1, 4), (4, 1), (33, 33), (120, 77), (77, 120)])
def test_oracle_factorisation_identity(m, n):
    A = np.random.default_rng(m * 1000 + n).uniform(-2, 2, (m, n))
    LU, ipiv = O.lu_partial_pivot(A)
    L, U = factors(LU)
    assert np.abs(L @ U - O.lu_apply_ipiv(A, ipiv)).max() <= 1e-12 * max(1.0, np.abs(A).max()) * max(m, n)
    assert np.all(np.abs(np.tril(LU[:, :min(m, n)], -1)) <= 1.0 + 1e-15)  # partial pivoting bounds |l| by 1


def test_oracle_no_pivot_on_diagonally_dominant():
    g = np.random.default_rng(3)
    A = g.uniform(-1, 1, (60, 60)) + 80 * np.eye(60)
    LU, ipiv = O.lu_partial_pivot(A, pivot=False)
    L, U = factors(LU)
    assert np.array_equal(ipiv, np.arange(1, 61))
    assert np.abs(L @ U - A).max() <= 1e-12 * 80


@pytest.mark.skipif(not REF_LIB.exists(), reason="oracle/_ref/libdarray_ref.so not built")
@pytest.mark.parametrize("m,n,bs", [(50, 50, 16), (70, 40, 16), (40, 70, 256), (129, 129, 32)])
def test_oracle_matches_reference_live(m, n, bs):
    lib = ctypes.CDLL(str(REF_LIB))
    fp, ip = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)
    lib.ref_lu.argtypes = [fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ip]
    A = np.asfortranarray(np.random.default_rng(m + n + bs).uniform(-2, 2, (m, n)).astype(np.float32))
    LUo, ipo = O.lu_partial_pivot(A)
    ipiv = np.zeros(min(m, n), np.int32)
    lib.ref_lu(A.ctypes.data_as(fp), m, n, bs, ipiv.ctypes.data_as(ip))
    assert np.array_equal(ipo, ipiv)
    assert np.abs(LUo - A).max() <= 2e-5 * np.abs(LUo).max()
