"""Golden fixtures for the LIBSVM reader: the reference's own read_input_file<T> (include/read_input.h:8-36,
compiled from its sources into oracle/_ref/libdarray_ref.so by oracle/build_ref.sh) run on the text cases of
tests/libsvm_cases.py.  Writes tests/golden/libsvm_reference.npz.

Run in the container that holds the reference checkout:
    ./oracle/build_ref.sh && python tests/golden/gen_libsvm_goldens.py
"""
from __future__ import annotations

import ctypes
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "tests"))
from libsvm_cases import cases  # noqa: E402

REF_LIB = ROOT / "oracle" / "_ref" / "libdarray_ref.so"
OUT = Path(__file__).resolve().parent / "libsvm_reference.npz"
FILL_X, FILL_Y = 7.0, 3.0  # entries the text does not name keep these


def reference_read(lib, text: bytes, n: int, d: int, dtype):
    fn = lib.ref_read_input_file_f32 if dtype == np.float32 else lib.ref_read_input_file_f64
    P = ctypes.POINTER(ctypes.c_float if dtype == np.float32 else ctypes.c_double)
    fn.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, P, P]
    X = np.full((n, d), FILL_X, dtype)
    Y = np.full(n, FILL_Y, dtype)
    with tempfile.NamedTemporaryFile(delete=False) as f:
        f.write(text)
        path = f.name
    try:
        fn(path.encode(), n, d, X.ctypes.data_as(P), Y.ctypes.data_as(P))
    finally:
        os.unlink(path)
    return X, Y


def main():
    lib = ctypes.CDLL(str(REF_LIB))
    out = {}
    for name, text, n, d in cases():
        out[f"{name}__text"] = np.frombuffer(text, np.uint8)
        out[f"{name}__nd"] = np.array([n, d])
        for tag, dt in (("f32", np.float32), ("f64", np.float64)):
            X, Y = reference_read(lib, text, n, d, dt)
            out[f"{name}__X_{tag}"] = X
            out[f"{name}__Y_{tag}"] = Y
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
