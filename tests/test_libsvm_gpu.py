"""The GPU LIBSVM reader (db200_libsvm_parse on device text, db200_read_libsvm from a file) against the CPU
restatement of the reference's read_input_file<T> (include/read_input.h:8-36), which
tests/test_libsvm_oracle.py pins bit for bit to the reference itself.

Bar: bit-identical X and y, as float and as double, and the same line count, on every case of
tests/libsvm_cases.py; text at unaligned device addresses; rows padded beyond d left untouched; the refused
inputs give DB200_ERR_INVALID (undefined in the reference) or DB200_ERR_UNSUPPORTED.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle.libsvm import read_input_file

sys.path.insert(0, str(Path(__file__).resolve().parent))
from libsvm_cases import ERROR_CASES, cases  # noqa: E402

pytestmark = pytest.mark.gpu

FILL_X, FILL_Y = 7.0, 3.0
CASES = cases()
UINT = {np.float32: np.uint32, np.float64: np.uint64}
ERR_INVALID, ERR_UNSUPPORTED = -1, -8


def oracle_read(text, n, d, dt):
    X = np.full((n, d), FILL_X, dt)
    Y = np.full(n, FILL_Y, dt)
    lines = read_input_file(text, n, d, X, Y, dt)
    return X, Y, lines


def gpu_parse(ctx, text, n, d, dt, offset=0, ldx=None):
    import torch
    from darray_optimizer_b200._lib import F32, F64
    ldx = ldx or d
    buf = torch.zeros(len(text) + offset + 1, dtype=torch.uint8, device="cuda")
    if text:
        buf[offset:offset + len(text)] = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()
    tdt = torch.float32 if dt == np.float32 else torch.float64
    X = torch.full((max(n, 1), ldx), FILL_X, dtype=tdt, device="cuda")
    Y = torch.full((max(n, 1),), FILL_Y, dtype=tdt, device="cuda")
    lines = ctx.libsvm_parse(buf.data_ptr() + offset, len(text), n, d, F32 if dt == np.float32 else F64,
                             X.data_ptr(), ldx, Y.data_ptr())
    ctx.sync()
    return X.cpu().numpy()[:n], Y.cpu().numpy()[:n], lines


def same_bits(a, b, dt):
    return a.shape == b.shape and np.array_equal(a.view(UINT[dt]), b.view(UINT[dt]))


@pytest.mark.parametrize("name,text,n,d", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("offset", [0, 3])
def test_parse_matches_oracle(gpu_ctx, name, text, n, d, dt, offset):
    Xo, Yo, lo = oracle_read(text, n, d, dt)
    Xg, Yg, lg = gpu_parse(gpu_ctx, text, n, d, dt, offset)
    assert lg == lo
    assert same_bits(Xg[:, :d], Xo, dt)
    assert same_bits(Yg, Yo, dt)


def test_parse_leaves_row_padding(gpu_ctx):
    name, text, n, d = CASES[0]
    Xo, Yo, _ = oracle_read(text, n, d, np.float32)
    Xg, Yg, _ = gpu_parse(gpu_ctx, text, n, d, np.float32, ldx=d + 5)
    assert same_bits(np.ascontiguousarray(Xg[:, :d]), Xo, np.float32)
    assert np.all(Xg[:, d:] == FILL_X)


def test_parse_c2_shaped_text(gpu_ctx):
    """4096 dense rows of 128 six-decimal values (the C2 point shape) plus a checksum of every value."""
    from darray_optimizer_b200.datagen import libsvm_text
    g = np.random.default_rng(3)
    n, d = 4096, 128
    X = g.random((n, d))
    y = np.where(g.random(n) < 0.5, 1.0, -1.0)
    text = libsvm_text(X, y, 6)
    Xo, Yo, lo = oracle_read(text, n, d, np.float32)
    Xg, Yg, lg = gpu_parse(gpu_ctx, text, n, d, np.float32)
    assert lg == lo == n
    assert same_bits(Xg, Xo, np.float32) and same_bits(Yg, Yo, np.float32)
    assert np.abs(Xg.astype(np.float64) - X).max() <= 5e-7 + 1e-7
    assert np.array_equal(Yg, y.astype(np.float32))


def test_parse_empty_inputs(gpu_ctx):
    assert gpu_parse(gpu_ctx, b"", 4, 3, np.float32)[2] == 0
    Xg, Yg, lg = gpu_parse(gpu_ctx, b"1 1:2\n", 0, 3, np.float32)
    assert lg == 0


@pytest.mark.parametrize("name,text,n,d", ERROR_CASES, ids=[c[0] for c in ERROR_CASES])
def test_parse_refuses(gpu_ctx, name, text, n, d):
    from darray_optimizer_b200._lib import DB200Error
    with pytest.raises(DB200Error) as e:
        gpu_parse(gpu_ctx, text, n, d, np.float32)
    want = ERR_INVALID if name in ("index_above_d", "blank_last_line") else ERR_UNSUPPORTED
    assert e.value.status == want
    assert "line" in str(e.value)


@pytest.mark.parametrize("name", ["dense_repr", "structure", "long_repeats"])
@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=["f32", "f64"])
def test_read_file_matches_oracle(gpu_ctx, tmp_path, name, dt):
    from darray_optimizer_b200._lib import F32, F64
    _, text, n, d = next(c for c in CASES if c[0] == name)
    path = tmp_path / f"{name}.libsvm"
    path.write_bytes(text)
    Xo, Yo, lo = oracle_read(text, n, d, dt)
    X = np.full((n, d), FILL_X, dt)
    Y = np.full(n, FILL_Y, dt)
    lines = gpu_ctx.read_libsvm(path, n, d, F32 if dt == np.float32 else F64, X.ctypes.data, d, Y.ctypes.data)
    assert lines == lo
    assert same_bits(X, Xo, dt) and same_bits(Y, Yo, dt)


def test_read_file_missing(gpu_ctx, tmp_path):
    from darray_optimizer_b200._lib import DB200Error, F32
    X = np.zeros((2, 2), np.float32)
    Y = np.zeros(2, np.float32)
    with pytest.raises(DB200Error) as e:
        gpu_ctx.read_libsvm(tmp_path / "absent.libsvm", 2, 2, F32, X.ctypes.data, 2, Y.ctypes.data)
    assert e.value.status == ERR_INVALID
