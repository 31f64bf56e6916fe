"""The reference's own test programs (tests/test3.cpp .. test7.cpp), unmodified, compiled against this build's
one-rank mirror headers (include/darray_b200/) and linked with libdarray_b200.so by oracle/build_ref.sh, run on
the GPU: code written against DArray's headers builds and runs on the product without source changes.

Checks per program, from what each prints:
  test3  recursive Cholesky of a 10 x 10 submatrix (runs to completion)
  test4  LU with partial pivoting at n = 512, bs = 64: fnorm(A - P L U) / fnorm(A) < 1e-5
  test5  matrix_multiply (T, N) and triangular_solve (L, U, T, N) on descriptors (runs to completion)
  test6  TSQR of a 10 x 3 matrix: from the printed A, R and Q (3 decimals), Q R = A and Q^T Q = I to 1e-2
  test7  one n x k block of K.O through tc_gemm (runs to completion)
The binaries come with the repository's reference build (absent without it: skipped)."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BIN = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "reftests"


def _run(name, *args):
    exe = BIN / name
    if not exe.exists():
        pytest.skip("the reference's test programs were not built here (oracle/build_ref.sh)")
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (name, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


def _matrices(text):
    """Blocks of numeric rows following a title line, from DArray's LMatrix::print."""
    blocks, cur, title = {}, None, None
    for line in text.splitlines():
        nums = re.findall(r"-?\d+\.\d+", line)
        if nums and len(nums) == len(line.split()):
            cur.append([float(x) for x in nums])
        else:
            title = line.strip()
            cur = []
            blocks[title] = cur
    return {k: np.array(v) for k, v in blocks.items() if v}


def test_reference_test3_recursive_cholesky():
    out = _run("test3")
    assert "cholesky" in out


def test_reference_test4_lu_backward_error():
    out = _run("test4", "-n", 512, "-b", 64)
    m = re.search(r"fnorm\(A-P\*L\*U\)/fnorm\(A\)=([0-9.eE+-]+)", out)
    assert m, out[-1000:]
    assert float(m.group(1)) < 1e-5


def test_reference_test5_multiply_and_triangular_solve():
    _run("test5")


def test_reference_test6_tsqr():
    mats = _matrices(_run("test6"))
    A, R, Q = mats["A"], mats["R"], mats["Q"]
    assert A.shape == (10, 3) and R.shape == (3, 3) and Q.shape == (10, 3)
    assert np.max(np.abs(Q @ R - A)) < 1e-2
    assert np.max(np.abs(Q.T @ Q - np.eye(3))) < 1e-2


def test_reference_test7_kernel_block_times_sketch():
    out = _run("test7", 4096, 64, 1024)
    assert "1 block of K*O takes" in out
