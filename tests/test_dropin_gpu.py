"""C++ drop-in: tests/cpp/test_dropin.cpp, written against DArray's headers (one-rank mirror in
include/darray_b200/) and the reference's dkernel.h symbols exported by libdarray_b200.so, run on the GPU."""
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

BIN = Path(__file__).resolve().parent / "cpp" / "_bin" / "test_dropin"


def test_cpp_dropin_program():
    if not BIN.exists():
        from darray_optimizer_b200 import build
        build.build()
    r = subprocess.run([str(BIN)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "ALL" in r.stdout and "CHECKS PASSED" in r.stdout
