"""Golden fixtures from the reference's own GPU kernel-block code, and its timing beside the drop-in symbols.

The reference computes kernel blocks and the sketch product only on the GPU (include/dkernel.cu: rbf_kernel,
tc_gemm; FP32, cuBLAS).  oracle/build_ref.sh compiles that file unmodified for sm_100a into
oracle/_ref/libdkernel_ref.so.  Run on a machine with a B200:

    python tests/golden/gen_reference_gpu_goldens.py [--out PATH]   # writes the fixtures
    python tests/golden/gen_reference_gpu_goldens.py --time         # times one 8192 x 8192 block

The fixtures (tests/golden/reference_gpu_goldens.npz by default) hold, for seeded inputs:
  * kblock_*: K = rbf_kernel(Xi, Xj, yi, yj, gamma), m = 200, n = 131, d = 20;
  * lra_*: Y = tc_gemm(rbf_kernel(X, X, y, y, gamma), Omega), one LRA block (include/dkernel.h:13-46) with
    n = 1536, d = 32, l = 48 on the two-class Gaussian generator.  tc_gemm overwrites its output for each
    8192-column block (beta = 0 every block), so fixtures stay at n <= 8192 where its result is the product.

--time runs one 8192 x 8192 block at d = 128, l = 528 through the reference (rbf_kernel then tc_gemm, host
buffers in and out) and through the product library's drop-in symbols of the same names and signatures on
the same host buffers, and prints one JSON line with seconds per block for each.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
REF_GPU_LIB = ROOT / "oracle" / "_ref" / "libdkernel_ref.so"
OUT = Path(__file__).resolve().parent / "reference_gpu_goldens.npz"
SEED = 20261203

_fp = ctypes.POINTER(ctypes.c_float)
_i, _f = ctypes.c_int, ctypes.c_float


def _p(a):
    return a.ctypes.data_as(_fp)


def load_reference():
    lib = ctypes.CDLL(str(REF_GPU_LIB))
    lib.ref_cuda_init.argtypes = []
    lib.ref_rbf_kernel.argtypes = [_i, _i, _i, _fp, _fp, _fp, _fp, _fp, _i, _f]
    lib.ref_tc_gemm.argtypes = [_i, _i, _i, _fp, _i, _fp, _i, _fp, _i, _f]
    lib.ref_cuda_init()
    return lib


def kblock_inputs():
    g = np.random.default_rng(SEED)
    m, n, d = 200, 131, 20
    Xi = g.standard_normal((m, d)).astype(np.float32)
    Xj = g.standard_normal((n, d)).astype(np.float32)
    yi = np.where(g.random(m) < 0.5, 1.0, -1.0).astype(np.float32)
    yj = np.where(g.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    return Xi, Xj, yi, yj, np.float32(0.7 / d)


def lra_inputs():
    g = np.random.default_rng(SEED + 1)
    n, d, l = 1536, 32, 48
    y = np.where(g.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    X = (g.standard_normal((n, d)) + 0.5 * y[:, None]).astype(np.float32)
    Omega = g.standard_normal((n, l)).astype(np.float32)
    return X, y, Omega, np.float32(1.0 / d)


def ref_rbf(lib, Xi, Xj, yi, yj, gamma):
    m, d = Xi.shape
    n = Xj.shape[0]
    xi, xj = np.asfortranarray(Xi), np.asfortranarray(Xj)
    K = np.zeros((m, n), np.float32, order="F")
    lib.ref_rbf_kernel(m, n, d, _p(xi), _p(xj), _p(np.ascontiguousarray(yi)), _p(np.ascontiguousarray(yj)),
                       _p(K), m, float(gamma))
    return K


def ref_gemm(lib, A, Bm):
    m, n = A.shape
    k = Bm.shape[1]
    a, b = np.asfortranarray(A), np.asfortranarray(Bm)
    C = np.zeros((m, k), np.float32, order="F")
    lib.ref_tc_gemm(m, k, n, _p(a), m, _p(b), n, _p(C), m, 1.0)
    return C


def make_fixtures(out: Path):
    lib = load_reference()
    Xi, Xj, yi, yj, gamma = kblock_inputs()
    K = ref_rbf(lib, Xi, Xj, yi, yj, gamma)
    X, y, Omega, gl = lra_inputs()
    Y = ref_gemm(lib, ref_rbf(lib, X, X, y, y, gl), Omega)
    np.savez_compressed(out, kblock_Xi=Xi, kblock_Xj=Xj, kblock_yi=yi, kblock_yj=yj, kblock_gamma=gamma,
                        kblock_K=K, lra_X=X, lra_y=y, lra_Omega=Omega, lra_gamma=gl, lra_Y=Y)
    print(f"wrote {out}")


def time_block(reps: int = 3):
    """One 8192 x 8192 block at d = 128, l = 528: reference rbf_kernel + tc_gemm against the product's
    drop-in symbols, same host buffers, wall time per block (both calls are synchronous)."""
    lib = load_reference()
    import darray_optimizer_b200._lib as L
    ours = L.load()
    o_rbf = getattr(ours, "_Z10rbf_kerneliiiiPfiS_iS_S_S_if")
    o_rbf.argtypes = [_i, _i, _i, _i, _fp, _i, _fp, _i, _fp, _fp, _fp, _i, _f]
    o_gemm = getattr(ours, "_Z7tc_gemmiiiiPfiS_iS_iff")
    o_gemm.argtypes = [_i, _i, _i, _i, _fp, _i, _fp, _i, _fp, _i, _f, _f]
    getattr(ours, "_Z9cuda_initv")()

    b, d, l = 8192, 128, 528
    g = np.random.default_rng(SEED + 2)
    X = np.asfortranarray(g.random((b, d), dtype=np.float32))
    y = np.where(g.random(b) < 0.5, 1.0, -1.0).astype(np.float32)
    Om = np.asfortranarray(g.standard_normal((b, l)).astype(np.float32))
    gamma = 0.5 / d
    K = np.zeros((b, b), np.float32, order="F")
    Y = np.zeros((b, l), np.float32, order="F")

    def run_ref():
        lib.ref_rbf_kernel(b, b, d, _p(X), _p(X), _p(y), _p(y), _p(K), b, gamma)
        lib.ref_tc_gemm(b, l, b, _p(K), b, _p(Om), b, _p(Y), b, 1.0)

    def run_ours():
        o_rbf(0, b, b, d, _p(X), b, _p(X), b, _p(y), _p(y), _p(K), b, gamma)
        o_gemm(0, b, l, b, _p(K), b, _p(Om), b, _p(Y), b, 1.0, 0.0)

    res = {}
    for name, fn in (("reference", run_ref), ("dropin", run_ours)):
        fn()  # warm-up: handles, allocations, module load
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
        res[name] = {"s_per_block": float(np.median(ts)), "Y": Y.copy()}
    flops = 2.0 * b * b * (d + l)
    rel = float(np.linalg.norm(res["dropin"]["Y"] - res["reference"]["Y"]) / np.linalg.norm(res["reference"]["Y"]))
    line = {"block": [b, b], "d": d, "l": l, "flops_per_block": flops, "blocks_per_c2_pass": (131072 // b) ** 2,
            "rel_fro_dropin_vs_reference": rel, "host_cores": os.cpu_count()}
    for name in ("reference", "dropin"):
        s = res[name]["s_per_block"]
        line[name] = {"s_per_block": s, "tflops": flops / s / 1e12, "c2_pass_s": s * (131072 // b) ** 2}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", type=Path, default=OUT)
    ap.add_argument("--time", action="store_true")
    a = ap.parse_args()
    if a.time:
        time_block()
    else:
        make_fixtures(a.out)


if __name__ == "__main__":
    main()
