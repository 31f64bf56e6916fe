"""Build libdarray_b200.so in-tree with nvcc for sm_100a.

Usage: python -m darray_optimizer_b200.build [--verbose]

The library lands in darray_optimizer_b200/lib/ so that it ships with the source tree; nothing is installed
elsewhere.  Objects are rebuilt only when a source or header is newer than the object.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libdarray_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "--expt-relaxed-constexpr", f"-I{ROOT / 'include'}", f"-I{CSRC}"]

SOURCES = sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))
HEADERS = sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").rglob("*.h")))


def _newest(paths):
    return max((p.stat().st_mtime for p in paths), default=0.0)


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    hdr_time = _newest(HEADERS)
    objs = []
    for src in SOURCES:
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_time):
            continue
        cmd = [NVCC, *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
        if src.suffix == ".cu":
            cmd += ["-Xptxas", "-v"] if verbose else []
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src.name}")
        if verbose and (r.stdout or r.stderr):
            sys.stderr.write(r.stdout + r.stderr)
    if force or not LIB.exists() or LIB.stat().st_mtime < _newest(objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-cudart", "static", "-lpthread", "-ldl",
               "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc link failed")
    build_cpp_tests(verbose)
    return LIB


CPP_TESTS = [ROOT / "tests" / "cpp" / "test_dropin.cpp"]
CPP_BIN = ROOT / "tests" / "cpp" / "_bin"


def build_cpp_tests(verbose: bool = False) -> None:
    """Compile the C++ drop-in tests (host code over include/darray_b200/ and the C ABI) next to their sources."""
    CPP_BIN.mkdir(exist_ok=True)
    hdr_time = _newest(HEADERS)
    for src in CPP_TESTS:
        out = CPP_BIN / src.stem
        if out.exists() and out.stat().st_mtime >= max(src.stat().st_mtime, hdr_time, LIB.stat().st_mtime):
            continue
        cmd = ["g++", "-O2", "-std=c++17", f"-I{ROOT / 'include'}", str(src), "-o", str(out), f"-L{LIBDIR}",
               "-ldarray_b200", "-Wl,-rpath,$ORIGIN/../../../darray_optimizer_b200/lib"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"g++ failed on {src.name}")


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(LIB)
