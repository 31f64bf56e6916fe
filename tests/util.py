"""Helpers shared by the GPU tests: numpy <-> torch device buffers with explicit column-major layout."""
import numpy as np


def dev(a, dtype=None):
    """Copy a numpy array to cuda:0 keeping its memory order (Fortran arrays stay column-major)."""
    import torch
    a = np.asarray(a)
    if dtype is not None:
        a = a.astype(dtype, copy=False)
    if a.ndim == 2 and a.flags.f_contiguous and not a.flags.c_contiguous:
        return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()  # stored transposed: same bytes
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def colmajor_empty(m, n, ld=None, dtype="float32"):
    """Device buffer for an m x n column-major matrix with leading dimension ld (returned as ld x n storage
    viewed as an (n, ld) torch tensor)."""
    import torch
    ld = ld or m
    return torch.zeros((n, ld), dtype=getattr(torch, dtype), device="cuda")


def colmajor_host(t, m):
    """Read an (n, ld) device buffer back as an m x n numpy array."""
    a = t.cpu().numpy()
    return np.asfortranarray(a[:, :m].T)


def ptr(t):
    return 0 if t is None else t.data_ptr()


def rel_fro(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64)) /
                 max(np.linalg.norm(np.asarray(b, np.float64)), 1e-300))
