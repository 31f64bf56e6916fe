"""CPU restatement of the integer-sliced FP64 Gram that the GPU computes on its int8 tensor cores -- TEST
INFRASTRUCTURE ONLY (tests/ may import it; the product never does).

The capacity matrix of the barrier's Woodbury solve is M = Z^T diag(w) Z (include/dbarrier.h:84-139 builds the
same operator Z Z^T + D implicitly for its PCG).  The GPU forms it by the Ozaki splitting scheme (Ozaki, Ogita,
Oishi, Rump, Numer. Algorithms 59, 2012): the rows are cut into chunks of 16384; in each chunk every column p of
Z~ = diag(sqrt(w)) Z is scaled by 2^-e with max |Z~[chunk, p]| < 2^e and cut into `ks` signed 7-bit digits by
truncation; the digit products with s + t <= ks + 1 are summed exactly in integers per chunk.  This module does
the same arithmetic with exact int64 matrix products, so the GPU result must equal it up to the FP64 rounding of
the final scaling and of the atomic additions.
"""
import numpy as np


def col_exponents(Zw):
    """e_p with max_i |Zw[i, p]| < 2^e_p (0 for an all-zero column)."""
    m = np.max(np.abs(Zw), axis=0)
    e = np.zeros(m.shape, dtype=np.int64)
    nz = m > 0
    e[nz] = np.frexp(m[nz])[1]  # m = f 2^e with f in [0.5, 1)
    return e


def digits(Zw, e, ks):
    """(ks, n, r) int64 digits d_s in [-127, 127] with Zw 2^-e = sum_s d_s 2^-7s + remainder."""
    x = np.ldexp(Zw, -e[None, :])
    out = np.empty((ks,) + Zw.shape, dtype=np.int64)
    for s in range(ks):
        y = x * 128.0
        d = np.trunc(y)
        out[s] = d.astype(np.int64)
        x = y - d
    return out


CHUNK = 16384


def sliced_gram(Z, w, ks=7, chunk=CHUNK):
    """M~ = sum_chunks sum_{s + t <= ks + 1} 2^(e_p + e_q - 7(s + t)) (D_s^T D_t)[p, q] in FP64 from exact int64
    products (Z: n x r, w: n); e and D per row chunk.  The whole r x r matrix is returned (it is symmetric)."""
    n, r = Z.shape
    total = np.zeros((r, r))
    for c0 in range(0, n, chunk):
        Zw = np.sqrt(w[c0:c0 + chunk])[:, None] * Z[c0:c0 + chunk]
        e = col_exponents(Zw)
        D = digits(Zw, e, ks)
        groups = []
        for g in range(ks):
            acc = np.zeros((r, r), dtype=np.int64)
            for s in range(g + 1):
                acc += D[s].T @ D[g - s]
            groups.append(acc)
        # fold the exact group sums the way the GPU does: Horner in 2^-7 from the smallest group
        v = np.zeros((r, r))
        for g in range(ks - 1, -1, -1):
            v = v * 2.0 ** -7 + groups[g].astype(np.float64)
        total += np.ldexp(v, (e[:, None] + e[None, :] - 14).astype(np.int64))
    return total
