"""Generate golden fixtures by running the reference's own code (compiled from its sources at one MPI rank by
oracle/build_ref.sh) on seeded inputs.  Writes tests/golden/reference_goldens.npz.

Run in the container that holds the reference checkout:
    ./oracle/build_ref.sh && python tests/golden/gen_reference_goldens.py

Known-answer inputs come from the reference's own tests: the min(i+1, j+1) matrix whose Cholesky factor is the
all-ones upper triangle (perftests/perftest_cholesky.cpp:46-53, 76-84) and test3's lower-triangular (1+i+j)
factor (tests/test3.cpp:24-46).
"""
from __future__ import annotations

import ctypes
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
REF_LIB = ROOT / "oracle" / "_ref" / "libdarray_ref.so"
OUT = Path(__file__).resolve().parent / "reference_goldens.npz"

fp = ctypes.POINTER(ctypes.c_float)
dp = ctypes.POINTER(ctypes.c_double)


def f32(a):
    return np.asfortranarray(a, dtype=np.float32)


def f64(a):
    return np.asfortranarray(a, dtype=np.float64)


def P(a):
    return a.ctypes.data_as(fp if a.dtype == np.float32 else dp)


def main():
    lib = ctypes.CDLL(str(REF_LIB))
    lib.ref_f.restype = ctypes.c_double
    lib.ref_gg.restype = ctypes.c_double
    lib.ref_f.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
    lib.ref_gg.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_double, ctypes.c_double]
    lib.ref_grad_phi.argtypes = [ctypes.c_int, dp, ctypes.c_double, ctypes.c_double, dp]
    lib.ref_hess_phi.argtypes = [ctypes.c_int, dp, ctypes.c_double, ctypes.c_double, dp]
    lib.ref_matrix_multiply_tn.argtypes = [fp, fp, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                           ctypes.c_float, ctypes.c_int]
    lib.ref_writemodel.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, ctypes.c_double,
                                   dp, dp, dp, ctypes.c_double, ctypes.c_int, ctypes.c_int]
    g = np.random.default_rng(20240607)
    out = {}

    # Cholesky KAT: A = min(i+1, j+1) -> upper factor of ones (perftest_cholesky.cpp).
    n = 300
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    A = f32(np.minimum(i + 1, j + 1))
    out["chol_min_A"] = A.copy()
    lib.ref_cholesky(P(A), n, 64, 0)
    out["chol_min_R_blocked"] = np.triu(A)
    A = f32(out["chol_min_A"])
    lib.ref_cholesky(P(A), n, 32, 1)
    out["chol_min_R_recursive"] = np.triu(A)

    # test3: m = lower-triangular (1+i+j); A = m m^T; recursive Cholesky, n = 10, bs = 4.
    n = 10
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    m = np.where(i >= j, 1 + i + j, 0).astype(np.float64)
    A = f32(m @ m.T)
    out["chol_test3_A"] = A.copy()
    lib.ref_cholesky(P(A), n, 4, 1)
    out["chol_test3_R"] = np.triu(A)

    # random SPD, both Cholesky variants
    n = 200
    B = g.standard_normal((n, n))
    A = f32(B @ B.T / n + np.eye(n))
    out["chol_spd_A"] = A.copy()
    lib.ref_cholesky(P(A), n, 48, 0)
    out["chol_spd_R_blocked"] = np.triu(A)

    # TSQR of a tall-skinny matrix
    Y = f32(g.standard_normal((500, 20)))
    out["tsqr_A"] = Y.copy()
    R = f32(np.zeros((20, 20)))
    lib.ref_tsqr(P(Y), 500, 20, P(R))
    out["tsqr_Q"] = Y
    out["tsqr_R"] = R

    # singular values
    C = f32(g.standard_normal((50, 50)))
    out["svd_A"] = C.copy()
    S = np.zeros(50, np.float32)
    lib.ref_svd(P(C), 50, P(S))
    out["svd_S"] = S

    # triangular solve U^T X = B
    U = np.triu(g.standard_normal((64, 64))) + 8 * np.eye(64)
    U = f32(U)
    Bm = f32(g.standard_normal((64, 7)))
    out["trsm_U"] = U.copy()
    out["trsm_B"] = Bm.copy()
    lib.ref_triangular_solve(P(U), P(Bm), 64, 7, 8)
    out["trsm_X"] = Bm

    # C = alpha A^T B + beta C
    Am = f32(g.standard_normal((100, 30)))
    Bm = f32(g.standard_normal((100, 20)))
    Cm = f32(g.standard_normal((30, 20)))
    out["mm_A"], out["mm_B"], out["mm_C"] = Am.copy(), Bm.copy(), Cm.copy()
    lib.ref_matrix_multiply_tn(P(Am), P(Bm), P(Cm), 100, 30, 20, ctypes.c_float(-1.0), ctypes.c_float(1.0), 16)
    out["mm_out"] = Cm

    # barrier functions (FP64)
    nb, kb, Cbox, t = 300, 20, 1.0, 3.0
    Z = f64(g.standard_normal((nb, kb)) * 0.3)
    a = f64(g.uniform(0.05, 0.95, nb))
    out["bar_Z"], out["bar_a"] = Z.copy(), a.copy()
    out["bar_C_t"] = np.array([Cbox, t])
    out["bar_f"] = np.array([lib.ref_f(nb, kb, P(a), P(Z))])
    out["bar_gg"] = np.array([lib.ref_gg(nb, kb, P(a), P(Z), Cbox, t)])
    gf = f64(np.zeros(nb))
    lib.ref_grad_f(nb, kb, P(Z), P(a), P(gf))
    out["bar_grad_f"] = gf
    gp = f64(np.zeros(nb))
    lib.ref_grad_phi(nb, P(a), Cbox, t, P(gp))
    out["bar_grad_phi"] = gp
    gr = f64(np.zeros(nb))
    lib.ref_grad(nb, P(gf), P(gp), P(gr))
    out["bar_grad"] = gr
    D = f64(np.zeros(nb))
    lib.ref_hess_phi(nb, P(a), Cbox, t, P(D))
    out["bar_D"] = D

    # pre_conjgrad, as written (system Z Z^T + D + n I, right-hand side e_1, start at a)
    npc, kpc = 120, 8
    Zp = f64(g.standard_normal((npc, kpc)))
    Dp = f64(g.uniform(0.5, 2.0, npc))
    Mp = f64(np.einsum("ij,ij->i", Zp, Zp))
    bp = f64(np.zeros(npc))
    bp[0] = 1.0
    ap = f64(g.uniform(0.1, 0.9, npc))
    xp = f64(np.zeros(npc))
    out["pcg_Z"], out["pcg_D"], out["pcg_M"], out["pcg_b"], out["pcg_a"] = Zp.copy(), Dp.copy(), Mp.copy(), bp.copy(), ap.copy()
    lib.ref_pre_conjgrad(npc, kpc, P(Zp), P(Mp), P(Dp), P(bp), P(ap), P(xp))
    out["pcg_x"] = xp

    # writemodel text
    nw, dw, kw, Cw = 40, 5, 4, 1.0
    Xw = np.where(g.random((nw, dw)) < 0.6, g.standard_normal((nw, dw)), 0.0)
    yw = np.where(g.random(nw) < 0.5, 1.0, -1.0)
    aw = np.where(g.random(nw) < 0.3, 0.0, g.uniform(0.0, Cw, nw))
    aw[:3] = Cw
    Zw = g.standard_normal((nw, kw)) * 0.2
    out["wm_X"], out["wm_y"], out["wm_a"], out["wm_Z"] = Xw, yw, aw, Zw
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "model")
        Xcm = f64(Xw.T)  # d x n column major = point-major
        lib.ref_writemodel(path.encode(), nw, dw, kw, P(f64(aw)), Cw, P(f64(Zw)), P(f64(yw)), P(Xcm), 0.25,
                           int(np.sum(yw == -1)), int(np.sum(yw == 1)))
        out["wm_text"] = np.frombuffer(open(path, "rb").read(), dtype=np.uint8)

    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)", file=sys.stderr)


if __name__ == "__main__":
    main()
