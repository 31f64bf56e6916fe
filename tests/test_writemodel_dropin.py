"""The drop-in writemodel (include/darray_b200/dbarrier.h, restating include/dbarrier.h:395-470) writes the same
model bytes as the oracle's writemodel -- which tests/test_oracle.py pins byte for byte to the reference's own --
on seeded inputs with free, margin and bounded support vectors and points without nonzero features; and with a
solved bias (the dual with y^T a = 0) the model's rho is -b.  Host code only: no GPU."""
import shutil
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "writemodel_dropin.cpp"


@pytest.fixture(scope="module")
def binary(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    out = tmp_path_factory.mktemp("wm") / "writemodel_dropin"
    lib = ROOT / "darray_optimizer_b200" / "lib"
    r = subprocess.run(["g++", "-O2", "-std=c++17", f"-I{ROOT / 'include'}", str(SRC), "-o", str(out),
                        f"-L{lib}", "-ldarray_b200", f"-Wl,-rpath,{lib}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return out


def _case(seed, n=300, d=9, k=7, C=2.0):
    g = np.random.default_rng(seed)
    a = g.uniform(0, C, n)
    a[g.random(n) < 0.3] = 0.0       # not support vectors
    a[g.random(n) < 0.2] = C         # bounded support vectors
    Z = g.standard_normal((n, k)) * 0.3
    y = np.where(g.random(n) < 0.5, 1.0, -1.0)
    X = np.round(g.standard_normal((n, d)), 3)
    X[g.random((n, d)) < 0.4] = 0.0  # sparse features
    X[5] = 0.0                       # a point without any nonzero feature
    a[5] = 0.5 * C
    return a, Z, y, X, C, 0.125


def _write_input(path, a, Z, y, X, C, gamma, bias, minus, plus):
    n, k = Z.shape
    d = X.shape[1]
    with open(path, "wb") as fh:
        fh.write(struct.pack("5i", n, d, k, minus, plus))
        fh.write(struct.pack("3d", C, gamma, bias))
        fh.write(np.ascontiguousarray(a, np.float64).tobytes())
        fh.write(np.asfortranarray(Z, np.float64).tobytes(order="F"))
        fh.write(np.ascontiguousarray(y, np.float64).tobytes())
        fh.write(np.ascontiguousarray(X, np.float64).tobytes())  # point-major: X[j, kk] at j*d + kk


@pytest.mark.parametrize("seed,bias", [(1, None), (2, None), (3, -0.731), (4, 1.25)])
def test_dropin_writemodel_bytes_match_oracle(binary, tmp_path, seed, bias):
    a, Z, y, X, C, gamma = _case(seed)
    minus, plus = int(np.sum(y == -1)), int(np.sum(y == 1))
    inp = tmp_path / "in.bin"
    _write_input(inp, a, Z, y, X, C, gamma, 0.0 if bias is None else bias, minus, plus)
    model = tmp_path / "model.txt"
    r = subprocess.run([str(binary), str(inp), str(model), "0" if bias is None else "1"], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    ref = tmp_path / "oracle.txt"
    res = O.writemodel(ref, a, C, Z, y, X, gamma, minus, plus, bias=bias)
    assert model.read_bytes() == ref.read_bytes()
    text = model.read_text()
    assert "rho %f" % (-res["b"]) in text
    if bias is not None:
        assert res["b"] == bias
    assert text.count("\n") == 9 + res["nSV"]
