"""Seeded synthetic workloads (Philox counter-based generator) standing in for the LIBSVM datasets the
reference's run scripts use (covtype, ijcnn1, SUSY, HIGGS; tests/README.md:31-143), which are not available.

Points are returned point-major (n x d float32, row i = point i), which is the byte layout of the reference's
DMatrix X (d x n column major, tests/testsvm.cpp:76).  Labels are +-1 float32 (read_input.h:20-22 maps every
label to +-1).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(seed))


@dataclass
class Workload:
    name: str
    X: np.ndarray            # n x d float32, point-major
    y: np.ndarray            # n float32 in {-1, +1}
    gamma: float
    rank: int                # target rank r
    oversample: int          # p; sketch width l = r + p
    power_iters: int         # q
    C: float                 # box constraint
    seed: int
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.X.shape[0]

    @property
    def d(self) -> int:
        return self.X.shape[1]

    @property
    def l(self) -> int:
        return self.rank + self.oversample

    def omega(self, seed_offset: int = 7919) -> np.ndarray:
        """Gaussian test matrix Omega (n x l, float32, Fortran/column-major order like DMatrix O)."""
        g = rng(self.seed + seed_offset)
        return np.asfortranarray(g.standard_normal((self.n, self.l), dtype=np.float32))


def two_gaussians(n: int = 4096, d: int = 32, seed: int = 1) -> Workload:
    """Config 1: two isotropic Gaussians N(+-0.5*1, I), labels by component; gamma = 1/d, r = 128 + 10, q = 1,
    C = 1."""
    g = rng(seed)
    y = np.where(g.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    X = (g.standard_normal((n, d)) + 0.5 * y[:, None]).astype(np.float32)
    return Workload("two_gaussians", X, y, 1.0 / d, 128, 10, 1, 1.0, seed)


def _two_gaussians_points(g, n, d):
    y = np.where(g.random(n) < 0.5, 1.0, -1.0).astype(np.float32)
    return (g.standard_normal((n, d)) + 0.5 * y[:, None]).astype(np.float32), y


def uniform_hyperplane(n: int = 131072, d: int = 128, seed: int = 2, flip: float = 0.05) -> Workload:
    """Config 2: x ~ U[0,1)^d float32; y = sign(w.(x - mean)) for a seeded w, 5% of labels flipped;
    gamma = 0.5/d, r = 512 + 16, q = 1, C = 10."""
    g = rng(seed)
    X = g.random((n, d), dtype=np.float32)
    w = g.standard_normal(d)
    s = (X.astype(np.float64) - X.mean(axis=0, dtype=np.float64)) @ w
    y = np.where(s >= 0, 1.0, -1.0)
    flips = g.random(n) < flip
    y[flips] = -y[flips]
    return Workload("uniform_hyperplane", X, y.astype(np.float32), 0.5 / d, 512, 16, 1, 10.0, seed,
                    meta={"w": w, "mean": X.mean(axis=0, dtype=np.float64), "flip": flip})


def sparse_binary(n: int = 262144, d: int = 123, seed: int = 3, p: float = 0.11) -> Workload:
    """Config 3: x_k ~ Bernoulli(0.11) in {0,1}; y = sign(w.x + b + eps), w ~ N(0,1) on a random 20% of the
    coordinates (0 elsewhere), eps ~ N(0, 0.5), b = -mean(w.x) so both classes appear; gamma = 0.05,
    r = 1024 + 16, C = 1."""
    g = rng(seed)
    X = (g.random((n, d)) < p).astype(np.float32)
    w = np.zeros(d)
    idx = g.choice(d, size=max(1, int(round(0.2 * d))), replace=False)
    w[idx] = g.standard_normal(idx.size)
    s = X.astype(np.float64) @ w
    b = -s.mean()
    y = np.where(s + b + g.normal(0.0, 0.5, n) >= 0, 1.0, -1.0).astype(np.float32)
    return Workload("sparse_binary", X, y, 0.05, 1024, 16, 1, 1.0, seed, meta={"b": b, "w": w, "p": p})


def _mixture_points(g, n, meta):
    comp = g.integers(0, meta["means"].shape[0], size=n)
    d = meta["means"].shape[1]
    X = np.empty((n, d), dtype=np.float64)
    z = g.standard_normal((n, d))
    for c in range(meta["means"].shape[0]):
        sel = comp == c
        if sel.any():
            X[sel] = meta["means"][c] + (z[sel] * meta["scales"][c]) @ meta["rotations"][c].T
    return X.astype(np.float32), meta["labels"][comp].astype(np.float32)


def mixture(n: int = 524288, d: int = 64, seed: int = 5, components: int = 32, scale_lo: float = 0.1,
            scale_hi: float = 3.0, mean_sd: float = 4.0) -> Workload:
    """Config 5: a mixture of `components` anisotropic Gaussians with equal weights.  Component c has mean
    ~ N(0, mean_sd^2 I), a random rotation (orthogonal factor of a Gaussian matrix) and per-axis scales log-uniform
    in [scale_lo, scale_hi]; its label is a seeded random sign.  gamma = 1/d, r = 2048 landmarks, C = 1."""
    g = rng(seed)
    means = g.standard_normal((components, d)) * mean_sd
    rot = np.empty((components, d, d))
    for c in range(components):
        q, r = np.linalg.qr(g.standard_normal((d, d)))
        rot[c] = q * np.sign(np.diag(r))[None, :]
    scales = np.exp(g.uniform(np.log(scale_lo), np.log(scale_hi), size=(components, d)))
    labels = np.where(g.random(components) < 0.5, 1.0, -1.0)
    meta = {"means": means, "rotations": rot, "scales": scales, "labels": labels}
    X, y = _mixture_points(g, n, meta)
    return Workload("mixture", X, y, 1.0 / d, 2048, 16, 1, 1.0, seed, meta=meta)


def held_out(w: Workload, n_test: int) -> tuple[np.ndarray, np.ndarray]:
    """Test points from the same distribution and labelling rule as `w` (same hyperplane / class means), drawn
    from an independent stream (seed + 1 of the Philox family)."""
    g = rng(w.seed + 1)
    d = w.d
    if w.name == "two_gaussians":
        return _two_gaussians_points(g, n_test, d)
    if w.name == "uniform_hyperplane":
        X = g.random((n_test, d), dtype=np.float32)
        s = (X.astype(np.float64) - w.meta["mean"]) @ w.meta["w"]
        y = np.where(s >= 0, 1.0, -1.0)
        flips = g.random(n_test) < w.meta["flip"]
        y[flips] = -y[flips]
        return X, y.astype(np.float32)
    if w.name == "sparse_binary":
        X = (g.random((n_test, d)) < w.meta["p"]).astype(np.float32)
        s = X.astype(np.float64) @ w.meta["w"] + w.meta["b"]
        y = np.where(s + g.normal(0.0, 0.5, n_test) >= 0, 1.0, -1.0).astype(np.float32)
        return X, y
    if w.name == "mixture":
        return _mixture_points(g, n_test, w.meta)
    raise ValueError(w.name)


CONFIGS = {
    "c1": two_gaussians,
    "c2": uniform_hyperplane,
    "c3": sparse_binary,
    "c5": mixture,
}


def make(name: str, **kw) -> Workload:
    return CONFIGS[name](**kw)


def libsvm_text(X: np.ndarray, y: np.ndarray, decimals: int = 6) -> bytes:
    """LIBSVM text "label 1:x 2:x ... d:x\\n" of dense points with 0 <= x < 10, every value written with
    `decimals` decimals ("%.{decimals}f"), labels "1" / "-1".  Built column slot by column slot with numpy, so a
    C2-sized file (131072 x 128, about 220 MB) takes a couple of seconds."""
    X = np.asarray(X, np.float64)
    n, d = X.shape
    if n == 0:
        return b""
    if X.min() < 0 or X.max() >= 9.5:
        raise ValueError("libsvm_text writes values in [0, 10) only")
    scale = 10 ** decimals
    q = np.rint(X * scale).astype(np.int64)  # value * 10^decimals, rounded
    vw = 2 + decimals                         # "D.ddd..."
    prefixes = [f" {k + 1}:".encode() for k in range(d)]
    width = 2 + sum(len(p) + vw for p in prefixes) + 1
    buf = np.full((n, width), ord(" "), np.uint8)
    pos = 0
    pos_lab = pos
    pos += 2
    neg = np.asarray(y) < 0
    buf[:, pos_lab] = np.where(neg, ord("-"), ord(" "))
    buf[:, pos_lab + 1] = ord("1")
    for k, p in enumerate(prefixes):
        buf[:, pos:pos + len(p)] = np.frombuffer(p, np.uint8)
        pos += len(p)
        v = q[:, k]
        buf[:, pos] = ord("0") + v // scale
        buf[:, pos + 1] = ord(".")
        frac = v % scale
        for j in range(decimals):
            buf[:, pos + 2 + decimals - 1 - j] = ord("0") + frac % 10
            frac //= 10
        pos += vw
    buf[:, pos] = ord("\n")
    return buf.tobytes()
