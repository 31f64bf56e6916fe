"""The LIBSVM reader's CPU restatement (oracle/libsvm.py) against the reference's own read_input_file<T>
(include/read_input.h:8-36): bit-identical X and Y, as float and as double, on every case of
tests/libsvm_cases.py.

Checked against the committed fixture tests/golden/libsvm_reference.npz (written by
tests/golden/gen_libsvm_goldens.py from the reference compiled into oracle/_ref), and against that library live
when it is built.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle.libsvm import LibsvmError, read_input_file

sys.path.insert(0, str(Path(__file__).resolve().parent))
from libsvm_cases import ERROR_CASES, cases  # noqa: E402

GOLD = Path(__file__).resolve().parent / "golden" / "libsvm_reference.npz"
REF_LIB = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libdarray_ref.so"
FILL_X, FILL_Y = 7.0, 3.0
CASES = cases()
UINT = {np.float32: np.uint32, np.float64: np.uint64}


def oracle_read(text, n, d, dt):
    X = np.full((n, d), FILL_X, dt)
    Y = np.full(n, FILL_Y, dt)
    lines = read_input_file(text, n, d, X, Y, dt)
    return X, Y, lines


def same_bits(a, b, dt):
    return a.shape == b.shape and np.array_equal(a.view(UINT[dt]), b.view(UINT[dt]))


@pytest.mark.parametrize("name,text,n,d", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("tag,dt", [("f32", np.float32), ("f64", np.float64)])
def test_oracle_matches_reference_fixture(name, text, n, d, tag, dt):
    g = np.load(GOLD)
    assert bytes(g[f"{name}__text"]) == text, "case text changed: regenerate the fixture"
    X, Y, _ = oracle_read(text, n, d, dt)
    assert same_bits(X, g[f"{name}__X_{tag}"], dt)
    assert same_bits(Y, g[f"{name}__Y_{tag}"], dt)


@pytest.mark.skipif(not REF_LIB.exists(), reason="oracle/_ref/libdarray_ref.so not built")
@pytest.mark.parametrize("name,text,n,d", CASES, ids=[c[0] for c in CASES])
def test_oracle_matches_reference_live(name, text, n, d):
    import ctypes
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    from gen_libsvm_goldens import reference_read
    lib = ctypes.CDLL(str(REF_LIB))
    for dt in (np.float32, np.float64):
        Xr, Yr = reference_read(lib, text, n, d, dt)
        X, Y, _ = oracle_read(text, n, d, dt)
        assert same_bits(X, Xr, dt) and same_bits(Y, Yr, dt)


def test_oracle_line_counts_and_untouched_entries():
    text = b"1 2:5\n-1 1:3\n"
    X, Y, lines = oracle_read(text, 4, 3, np.float32)
    assert lines == 2
    assert X[0].tolist() == [FILL_X, 5.0, FILL_X] and X[1].tolist() == [3.0, FILL_X, FILL_X]
    assert Y.tolist() == [1.0, -1.0, FILL_Y, FILL_Y]


@pytest.mark.parametrize("name,text,n,d", ERROR_CASES, ids=[c[0] for c in ERROR_CASES])
def test_oracle_refuses_undefined_or_unsupported_input(name, text, n, d):
    with pytest.raises(LibsvmError):
        oracle_read(text, n, d, np.float32)


def test_libsvm_text_writer_round_trips():
    """datagen.libsvm_text (the bench's C2-as-text writer) against the oracle reader: every value comes back as
    the float32 of its six-decimal rounding, every label as +-1, one line per point."""
    from darray_optimizer_b200.datagen import libsvm_text
    g = np.random.default_rng(5)
    n, d = 300, 17
    X = g.random((n, d))
    X[0, 0], X[1, 1] = 0.0, 9.4999994  # the ends of the writer's [0, 10) range
    y = np.where(g.random(n) < 0.5, 1.0, -1.0)
    text = libsvm_text(X, y, 6)
    assert text.count(b"\n") == n
    Xo = np.full((n, d), FILL_X, np.float32)
    Yo = np.full(n, FILL_Y, np.float32)
    assert read_input_file(text, n, d, Xo, Yo, np.float32) == n
    expect = np.array([[float(f"{v:.6f}") for v in row] for row in X], dtype=np.float32)
    assert np.array_equal(Xo, expect)
    assert np.array_equal(Yo, y.astype(np.float32))
