"""CPU checks of the C ABI boundary: the shared library loads and exports every function declared in
include/darray_b200.h (no compute calls: there is no GPU here)."""
import ctypes
import subprocess

from darray_optimizer_b200 import _lib


def test_library_loads():
    lib = _lib.load()
    assert isinstance(lib, ctypes.CDLL)


def test_every_header_function_is_exported():
    names = _lib.header_functions()
    assert "db200_rbf_sketch" in names and "db200_create" in names
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in names if n not in exported]
    assert not missing, missing


def test_bindings_cover_header():
    assert set(_lib.header_functions()) <= set(_lib.SIGNATURES)
