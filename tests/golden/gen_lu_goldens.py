"""Golden fixtures for the LU factorisation: the reference's own lu_factorize_partial_pivot<float>
(include/lapack_like.h:179-279, compiled from its sources at one MPI rank into oracle/_ref/libdarray_ref.so by
oracle/build_ref.sh) on seeded uniform(-2, 2) matrices, as in perftests/perftest_lu.cpp.  Writes
tests/golden/lu_reference.npz.

Run in the container that holds the reference checkout:
    ./oracle/build_ref.sh && python tests/golden/gen_lu_goldens.py
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
REF_LIB = ROOT / "oracle" / "_ref" / "libdarray_ref.so"
OUT = Path(__file__).resolve().parent / "lu_reference.npz"
CASES = [(64, 64, 16), (97, 60, 32), (45, 130, 16), (200, 200, 256)]  # m, n, outer block bs


def main():
    lib = ctypes.CDLL(str(REF_LIB))
    fp, ip = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)
    lib.ref_lu.argtypes = [fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ip]
    g = np.random.default_rng(20261203)
    out = {}
    for k, (m, n, bs) in enumerate(CASES):
        A = np.asfortranarray(g.uniform(-2, 2, (m, n)).astype(np.float32))
        out[f"c{k}_A"] = A.copy()
        ipiv = np.zeros(min(m, n), np.int32)
        lib.ref_lu(A.ctypes.data_as(fp), m, n, bs, ipiv.ctypes.data_as(ip))
        out[f"c{k}_LU"] = A
        out[f"c{k}_ipiv"] = ipiv
        out[f"c{k}_mnb"] = np.array([m, n, bs])
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
