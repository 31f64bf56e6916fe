"""The FP64 oracle against fixtures produced by the reference's own GPU kernel-block code
(include/dkernel.cu: rbf_kernel, tc_gemm), generated on a B200 by tests/golden/gen_reference_gpu_goldens.py.

Tolerances: kernel block max |dK| <= 1e-5; LRA block (rbf_kernel then tc_gemm) relative Frobenius error
<= 1e-5.  The reference computes in FP32 (cuBLAS GEMM distances, __expf); the oracle in FP64.
"""
from pathlib import Path

import numpy as np

from oracle import oracle as O

GOLD = Path(__file__).resolve().parent / "golden" / "reference_gpu_goldens.npz"


def test_oracle_rbf_block_matches_reference_gpu():
    g = np.load(GOLD)
    K = O.rbf_block(g["kblock_Xi"], g["kblock_Xj"], g["kblock_yi"], g["kblock_yj"], float(g["kblock_gamma"]))
    assert K.shape == g["kblock_K"].shape
    assert np.max(np.abs(K - g["kblock_K"])) <= 1e-5
    # the reference's identities: |K| <= 1 and the labels' signs
    assert np.all(np.abs(g["kblock_K"]) <= 1.0 + 1e-6)
    assert np.array_equal(np.sign(g["kblock_K"]), np.sign(np.outer(g["kblock_yi"], g["kblock_yj"])))


def test_oracle_sketch_matches_reference_gpu_lra_block():
    g = np.load(GOLD)
    X, y, Om = g["lra_X"], g["lra_y"], g["lra_Omega"]
    Y = O.sketch(X, X, y, y, Om, float(g["lra_gamma"]))
    ref = g["lra_Y"].astype(np.float64)
    assert Y.shape == ref.shape
    assert np.linalg.norm(Y - ref) <= 1e-5 * np.linalg.norm(ref)
