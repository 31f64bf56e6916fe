"""CPU oracle for the learned-landmark path (test infrastructure only: tests, smoke() and bench.py's CPU
baseline may use it; the product never calls it).

The reference has no landmark method (it always sketches with a Gaussian Omega, include/dkernel.h:13-46), so
this file restates, in FP64 numpy, exactly what darray_optimizer_b200/csrc/landmarks.cu computes:

* knn_distance: distance to the k-th nearest of a reference subset, a point never its own neighbour;
* leverage_features: [x, ||x||, knn];
* MLP forward / backward with the GPU's bf16 roundings (standardised input, each hidden activation and every
  weight rounded to bf16, round-to-nearest-even), FP64 arithmetic otherwise; Adam (beta1 0.9, beta2 0.999,
  eps 1e-8);
* ridge leverage lev_i = z_i^T (Z^T Z + lambda I)^-1 z_i;
* Gumbel keys from the splitmix64 finaliser (Vigna) of a per-index counter;
* the Nystrom factor Z = C R^-1, C = diag(y) K(:, L) diag(y_L), R^T R = C(L, :) + nu I, and the sampled
  residual ||Q(:, S) - Z Z(S, :)^T||_F / ||Q(:, S)||_F.

Parity is not pinned to the reference (there is nothing to pin it to); the MLP gradient is pinned by central
finite differences of this oracle's own loss in tests/test_landmarks_oracle.py.
"""
from __future__ import annotations

import numpy as np

# ------------------------------------------------------------------ features


def knn_distance(X: np.ndarray, ref_idx: np.ndarray, k: int) -> np.ndarray:
    X = np.asarray(X, dtype=np.float64)
    R = X[ref_idx]
    n = X.shape[0]
    out = np.empty(n)
    for i0 in range(0, n, 2048):
        Xi = X[i0:i0 + 2048]
        D = (Xi * Xi).sum(1)[:, None] + (R * R).sum(1)[None, :] - 2.0 * Xi @ R.T
        D = np.maximum(D, 0.0)
        rows = np.arange(i0, i0 + Xi.shape[0])
        D[rows[:, None] == ref_idx[None, :]] = np.inf
        out[i0:i0 + Xi.shape[0]] = np.sqrt(np.partition(D, k - 1, axis=1)[:, k - 1])
    return out


def leverage_features(X: np.ndarray, knn: np.ndarray) -> np.ndarray:
    X = np.asarray(X, dtype=np.float64)
    return np.concatenate([X, np.linalg.norm(X, axis=1, keepdims=True), np.asarray(knn, np.float64)[:, None]], axis=1)


# ------------------------------------------------------------------ bf16 rounding


def bf16(x) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even) and return as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    bias = ((u >> 16) & 1) + 0x7FFF
    r = ((u + bias) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


# ------------------------------------------------------------------ MLP


def mlp_layout(in_dim: int, width: int, hidden: int):
    """[(w_offset, b_offset, fan_in, fan_out)] in the flat parameter order of db200_mlp."""
    out, off = [], 0
    for l in range(hidden + 1):
        fi = in_dim if l == 0 else width
        fo = 1 if l == hidden else width
        out.append((off, off + fi * fo, fi, fo))
        off += fi * fo + fo
    return out, off


def _unpack(params, layout):
    Ws, bs = [], []
    for ow, ob, fi, fo in layout:
        Ws.append(np.asarray(params[ow:ow + fi * fo], np.float64).reshape(fo, fi))
        bs.append(np.asarray(params[ob:ob + fo], np.float64))
    return Ws, bs


def mlp_forward(params, F, mean, scale, width, hidden, round_bf16=True):
    """Returns (out, activations); activations[0] is the standardised input, [l] the output of hidden layer l."""
    F = np.asarray(F, np.float64)
    layout, _ = mlp_layout(F.shape[1], width, hidden)
    Ws, bs = _unpack(params, layout)
    rnd = bf16 if round_bf16 else (lambda v: np.asarray(v, np.float64))
    h = rnd((F - np.asarray(mean, np.float64)) * np.asarray(scale, np.float64))
    acts = [h]
    for l in range(hidden):
        h = rnd(np.maximum(h @ rnd(Ws[l]).T + bs[l], 0.0))
        acts.append(h)
    out = h @ rnd(Ws[hidden]).T + bs[hidden]
    return out[:, 0], acts


def mlp_loss_grad(params, F, target, mean, scale, width, hidden, round_bf16=True):
    """0.5 mean (out - t)^2 and its gradient (flat, the db200_mlp order); the backward pass uses the same rounded
    weights and activations as the forward pass, as the GPU does."""
    F = np.asarray(F, np.float64)
    m = F.shape[0]
    layout, npar = mlp_layout(F.shape[1], width, hidden)
    Ws, bs = _unpack(params, layout)
    rnd = bf16 if round_bf16 else (lambda v: np.asarray(v, np.float64))
    out, acts = mlp_forward(params, F, mean, scale, width, hidden, round_bf16)
    r = out - np.asarray(target, np.float64)
    loss = 0.5 * float(np.mean(r * r))
    g = np.zeros(npar)
    dY = (r / m)[:, None]
    for l in range(hidden, -1, -1):
        ow, ob, fi, fo = layout[l]
        g[ow:ow + fi * fo] = (dY.T @ acts[l]).ravel()
        g[ob:ob + fo] = dY.sum(0)
        if l > 0:
            dY = (dY @ rnd(Ws[l])) * (acts[l] > 0)
    return loss, g


def adam(params, grad, m1, m2, step, lr):
    """One Adam update (step counts from 1); returns (params, m1, m2)."""
    m1 = 0.9 * m1 + 0.1 * grad
    m2 = 0.999 * m2 + 0.001 * grad * grad
    c1 = 1.0 / (1.0 - 0.9 ** step)
    c2 = 1.0 / (1.0 - 0.999 ** step)
    return params - lr * (m1 * c1) / (np.sqrt(m2 * c2) + 1e-8), m1, m2


# ------------------------------------------------------------------ leverage, selection


def ridge_leverage(Z: np.ndarray, lam: float) -> np.ndarray:
    Z = np.asarray(Z, np.float64)
    G = Z.T @ Z + lam * np.eye(Z.shape[1])
    return np.einsum("ij,ij->i", Z, np.linalg.solve(G, Z.T).T)


_M64 = (1 << 64) - 1


def _mix64(z: np.ndarray) -> np.ndarray:
    z = z.astype(np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def gumbel_keys(logits: np.ndarray, seed: int) -> np.ndarray:
    n = logits.shape[0]
    with np.errstate(over="ignore"):
        ctr = (np.uint64((seed * 0x9E3779B97F4A7C15) & _M64) + np.arange(n, dtype=np.uint64) + np.uint64(1))
    h = _mix64(ctr)
    u = ((h >> np.uint64(11)).astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)
    return (np.asarray(logits, np.float32) + (-np.log(-np.log(u))).astype(np.float32)).astype(np.float32)


def topk_indices(keys: np.ndarray, k: int) -> np.ndarray:
    return np.sort(np.argsort(-np.asarray(keys, np.float64), kind="stable")[:k])


# ------------------------------------------------------------------ Nystrom factor, residual


def rbf_q(Xi, Xj, yi, yj, gamma) -> np.ndarray:
    Xi = np.asarray(Xi, np.float64)
    Xj = np.asarray(Xj, np.float64)
    D = (Xi * Xi).sum(1)[:, None] + (Xj * Xj).sum(1)[None, :] - 2.0 * Xi @ Xj.T
    return np.asarray(yi, np.float64)[:, None] * np.exp(-gamma * np.maximum(D, 0.0)) * np.asarray(yj, np.float64)[None, :]


def landmark_factor(X, y, gamma, idx):
    """Z = C R^-1 with C = diag(y) K(:, L) diag(y_L), R^T R = C(L, :) + nu I (nu = 1e-7 tr / r, x10 until SPD)."""
    idx = np.asarray(idx)
    C = rbf_q(X, X[idx], y, y[idx], gamma)
    W = C[idx]
    W = 0.5 * (W + W.T)
    r = len(idx)
    nu = 1e-7 * max(np.trace(W), 1e-300) / r
    for _ in range(12):
        try:
            R = np.linalg.cholesky(W + nu * np.eye(r)).T
            break
        except np.linalg.LinAlgError:
            nu *= 10.0
    else:
        raise np.linalg.LinAlgError("landmark_factor: not positive definite")
    return np.linalg.solve(R.T, C.T).T, nu


def residual_estimate(X, y, gamma, Z, sample_idx) -> float:
    S = np.asarray(sample_idx)
    Qs = rbf_q(X, X[S], y, y[S], gamma)
    T = np.asarray(Z, np.float64) @ np.asarray(Z, np.float64)[S].T
    return float(np.linalg.norm(Qs - T) / np.linalg.norm(Qs))
