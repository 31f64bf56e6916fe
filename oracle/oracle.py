"""FP64 CPU oracle for DArray's kernel-SVM hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this module, and only as the
checker or the timed CPU baseline; the product (darray_optimizer_b200 + libdarray_b200.so) never calls it.

It restates, in float64 numpy, the reference rushah05/DArray_Optimizer with its known defects corrected
(each correction is named where it is made):

  rbf_block          include/dkernel.cu:102-129 (vecnorm, rbf), :151-178 (GEMM-form distances, tiles)
  sketch (LRA)       include/dkernel.h:13-46 + include/dkernel.cu:194-231 (tc_gemm)
  knorm              include/dkernel.h:50-76
  householder_qr     include/lapack_like.h:283-379 (tall_skinny_qr_factorize at one rank)
  cholqr2            CholeskyQR2 (Yamamoto et al. 2015) built from lapack_like.h:10-56's Cholesky
  cholesky_upper     include/lapack_like.h:10-56 (cholesky_factorize, 'U')
  trsm_lutn          include/blas_like.h:96-127 (triangular_solve L,U,T,N)
  matmul_tn          include/blas_like.h:63-93 (matrix_multiply T,N)
  svd_values         include/lapack_like.h:389-413 (svd -> singular values only)
  f, gg, grad_f, grad_phi, grad, hess_phi   include/dbarrier.h:14-81
  pre_conjgrad       include/dbarrier.h:84-139 (kept verbatim in meaning, for pinning against the reference)
  newton_smw         replaces pre_conjgrad on the Newton path (see below)
  svm_barrier        tests/testsvm.cpp:192-321
  writemodel         include/dbarrier.h:395-470

Corrections relative to the reference (tests/testsvm.cpp, include/dkernel.h):
  1. LRA covers every (i, j) block (the reference returns after the first, dkernel.h:43) and accumulates the
     sketch over j (tc_gemm zeroes C and ignores beta, dkernel.cu:201).
  2. Knorm computes ||K - Z Z^T||_F / ||K||_F (the reference measures ||Z Z^T|| and overwrites, dkernel.h:67-72).
  3. The low-rank factor is Z = Q R^T with R^T R = Q^T K Q + nu I, so Z Z^T = Q (Q^T K Q) Q^T up to the shift
     (the reference scales Q by the singular values, testsvm.cpp:149-170).
  4. The Newton step solves (Z Z^T + diag(D)) s = -grad (Sherman-Morrison-Woodbury on the r x r capacity
     matrix I + Z^T D^-1 Z); the reference solves (Z Z^T + D + n I) x = e_1 by PCG (dbarrier.h:84-139,
     testsvm.cpp:232).
  5. The line search keeps 0 < a < C by capping the step at 0.99 of the distance to the box (the reference
     evaluates log of negative numbers, testsvm.cpp:275-288).
  6. Barrier stop at 2n/t < tol*|f(a)| with tol = 1e-6 (the reference uses 1e-5, testsvm.cpp:314).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

F64 = np.float64


# ----------------------------------------------------------------------------------------------- kernel
def row_norms(X: np.ndarray) -> np.ndarray:
    """vecnorm (include/dkernel.cu:102-114): s_i = sum_k x_ik^2."""
    X = np.asarray(X, F64)
    return np.einsum("ij,ij->i", X, X)


def rbf_block(Xi, Xj, yi=None, yj=None, gamma=1.0) -> np.ndarray:
    """K_ab = y_a y_b exp(-gamma (s_a + s_b - 2 x_a.x_b)), GEMM form as in include/dkernel.cu:116-129 and
    :160-169 (Xi and Xj are point-major m x d / n x d).  Squared distances are clamped at 0 (round-off near the
    diagonal can make them slightly negative)."""
    Xi = np.asarray(Xi, F64)
    Xj = np.asarray(Xj, F64)
    D2 = row_norms(Xi)[:, None] + row_norms(Xj)[None, :] - 2.0 * (Xi @ Xj.T)
    np.maximum(D2, 0.0, out=D2)
    K = np.exp(-gamma * D2)
    if yi is not None:
        K *= np.asarray(yi, F64)[:, None]
    if yj is not None:
        K *= np.asarray(yj, F64)[None, :]
    return K


def sketch(Xi, Xj, yi, yj, Omega, gamma, block: int = 2048) -> np.ndarray:
    """Y = diag(yi) K(Xi, Xj) diag(yj) Omega, streaming row blocks of K (include/dkernel.h:13-46 with
    correction 1).  Omega is n x l; Y is m x l."""
    Omega = np.asarray(Omega, F64)
    m = Xi.shape[0]
    Y = np.empty((m, Omega.shape[1]), F64)
    for i in range(0, m, block):
        Ki = rbf_block(Xi[i:i + block], Xj, None if yi is None else yi[i:i + block], yj, gamma)
        Y[i:i + block] = Ki @ Omega
    return Y


def knorm(X, y, Z, gamma, block: int = 2048) -> tuple[float, float, float]:
    """(||K||_F, ||K - Z Z^T||_F, ratio) with K = diag(y) K(X, X) diag(y) (include/dkernel.h:50-76 with
    correction 2)."""
    Z = np.asarray(Z, F64)
    kk = 0.0
    rr = 0.0
    for i in range(0, X.shape[0], block):
        Ki = rbf_block(X[i:i + block], X, y[i:i + block], y, gamma)
        kk += float(np.sum(Ki * Ki))
        R = Ki - Z[i:i + block] @ Z.T
        rr += float(np.sum(R * R))
    return math.sqrt(kk), math.sqrt(rr), math.sqrt(rr / kk)


# ----------------------------------------------------------------------------------------------- dense LA
def cholesky_upper(A: np.ndarray) -> np.ndarray:
    """Upper Cholesky factor R (A = R^T R), as cholesky_factorize(A, 'U', ...) (include/lapack_like.h:10-56)."""
    return np.linalg.cholesky(np.asarray(A, F64)).T


def trsm_lutn(R: np.ndarray, B: np.ndarray) -> np.ndarray:
    """X = R^-T B for upper R: triangular_solve("L","U","T","N") (include/blas_like.h:96-127)."""
    import scipy.linalg as sl
    return sl.solve_triangular(np.asarray(R, F64), np.asarray(B, F64), trans="T", lower=False)


def matmul_tn(A: np.ndarray, B: np.ndarray, C: np.ndarray | None = None, alpha=1.0, beta=0.0) -> np.ndarray:
    """C = alpha A^T B + beta C: matrix_multiply("T","N") (include/blas_like.h:63-93)."""
    out = alpha * (np.asarray(A, F64).T @ np.asarray(B, F64))
    if C is not None and beta != 0.0:
        out += beta * np.asarray(C, F64)
    return out


def householder_qr(Y: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Explicit thin Q and R of a tall-skinny matrix: tall_skinny_qr_factorize at one rank
    (include/lapack_like.h:283-379: local geqrf, QR of the stacked R, ormqr to form Q)."""
    Q, R = np.linalg.qr(np.asarray(Y, F64), mode="reduced")
    return Q, R


def cholqr2(Y: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """CholeskyQR2: W = Y^T Y, R1 = chol(W), Q1 = Y R1^-1, then once more on Q1.  Returns (Q, R2 R1).
    When the first Gram is numerically singular, shifted CholeskyQR3 (Fukaya et al. 2020): the first pass
    factors W + s I with s = 11 (n l + l (l + 1)) u trace(W), followed by two plain passes."""
    import scipy.linalg as sl
    Y = np.asarray(Y, F64)
    n, l = Y.shape

    def one(A, shift=0.0):
        W = A.T @ A
        if shift:
            W = W + shift * np.trace(W) * np.eye(l)
        R = cholesky_upper(W)
        return sl.solve_triangular(R, A.T, trans="T", lower=False).T, R

    try:
        Q1, R1 = one(Y)
        shifted = False
    except np.linalg.LinAlgError:
        Q1, R1 = one(Y, 11.0 * (n * l + l * (l + 1)) * np.finfo(F64).eps / 2)
        shifted = True
    Q, R2 = one(Q1)
    R = R2 @ R1
    if shifted:
        Q, R3 = one(Q)
        R = R3 @ R
    return Q, R


def sign_fix(Q: np.ndarray, R: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Flip column signs so that diag(R) >= 0 (makes Householder and Cholesky QR comparable)."""
    s = np.sign(np.diag(R))
    s[s == 0] = 1.0
    return Q * s[None, :], R * s[:, None]


def svd_values(C: np.ndarray) -> np.ndarray:
    """Singular values, descending: svd (include/lapack_like.h:389-413 returns only S)."""
    return np.linalg.svd(np.asarray(C, F64), compute_uv=False)


def shifted_cholesky(C: np.ndarray, rel_shift: float = 1e-7, tries: int = 12) -> tuple[np.ndarray, float]:
    """Upper R with R^T R = C + nu I, nu = rel_shift * trace(C) / l, increased x10 until positive definite."""
    C = 0.5 * (np.asarray(C, F64) + np.asarray(C, F64).T)
    l = C.shape[0]
    nu = rel_shift * max(np.trace(C), 1e-300) / l
    for _ in range(tries):
        try:
            return np.linalg.cholesky(C + nu * np.eye(l)).T, nu
        except np.linalg.LinAlgError:
            nu *= 10.0
    raise np.linalg.LinAlgError("shifted Cholesky failed")


# ----------------------------------------------------------------------------------------------- low rank
@dataclass
class LowRank:
    Z: np.ndarray
    Q: np.ndarray
    C: np.ndarray
    nu: float
    passes: int


def low_rank_factor(X, y, Omega, gamma, power_iters=1, orth="cholqr2", block=2048) -> LowRank:
    """Randomised range finder with power iteration and the Q C Q^T core (tests/testsvm.cpp:86-170 with
    correction 3): Y = K Omega; Q = orth(Y); q times {Y = K Q; Q = orth(Y)}; C = Q^T K Q; Z = Q R^T."""
    orth_fn = cholqr2 if orth == "cholqr2" else householder_qr
    Y = sketch(X, X, y, y, Omega, gamma, block)
    Q, R = sign_fix(*orth_fn(Y))
    passes = 1
    for _ in range(power_iters):
        Y = sketch(X, X, y, y, Q, gamma, block)
        Q, R = sign_fix(*orth_fn(Y))
        passes += 1
    KQ = sketch(X, X, y, y, Q, gamma, block)
    passes += 1
    C = Q.T @ KQ
    Rc, nu = shifted_cholesky(C)
    Z = Q @ Rc.T
    return LowRank(Z=Z, Q=Q, C=0.5 * (C + C.T), nu=nu, passes=passes)


# ----------------------------------------------------------------------------------------------- barrier
def f(a, Z) -> float:
    """f(a) = 0.5 a^T Z Z^T a - 1^T a (include/dbarrier.h:14-35)."""
    w = Z.T @ a
    return 0.5 * float(w @ w) - float(np.sum(a))


def gg(a, Z, C, t) -> float:
    """f(a) - (1/t) sum(log a + log(C - a)) (include/dbarrier.h:38-45)."""
    with np.errstate(invalid="ignore", divide="ignore"):
        lg = float(np.sum(np.log(a) + np.log(C - a))) / t
    return f(a, Z) - lg


def grad_f(Z, a) -> np.ndarray:
    """Z Z^T a - 1 (include/dbarrier.h:48-57)."""
    return Z @ (Z.T @ a) - 1.0


def grad_phi(a, C, t) -> np.ndarray:
    """(-1/a + 1/(C - a)) / t (include/dbarrier.h:60-65)."""
    return (-1.0 / a + 1.0 / (C - a)) / t


def grad(gradf, gradphi) -> np.ndarray:
    """include/dbarrier.h:68-73."""
    return gradf + gradphi


def hess_phi(a, C, t) -> np.ndarray:
    """D = (1/a^2 + 1/(C - a)^2) / t (include/dbarrier.h:76-81)."""
    return (1.0 / (a * a) + 1.0 / ((C - a) * (C - a))) / t


def pre_conjgrad(Z, M, D, b, a, tol=1e-2, max_iter=100000) -> tuple[np.ndarray, int]:
    """Jacobi-preconditioned CG on (Z Z^T + diag(D) + n I) x = b starting from x = a, as written in
    include/dbarrier.h:84-139 (kept for pinning against the reference; not used on the Newton path)."""
    n = Z.shape[0]
    x = np.array(a, F64)
    r = b - (Z @ (Z.T @ x) + D * x + n * x)
    z = r / M
    p = z.copy()
    rsold = float(r @ z)
    it = 0
    while np.linalg.norm(r) > tol and it < max_iter:
        Ap = Z @ (Z.T @ p) + D * p + n * p
        alpha = rsold / float(p @ Ap)
        x += alpha * p
        r -= alpha * Ap
        z = r / M
        rsnew = float(r @ z)
        p = z + (rsnew / rsold) * p
        rsold = rsnew
        it += 1
    return x, it


def lu_partial_pivot(A, pivot=True) -> tuple[np.ndarray, np.ndarray]:
    """LU with partial pivoting, restated from lu_factorize_partial_pivot / lu_factorize_unblocked
    (include/lapack_like.h:179-279) in FP64: for each column j the pivot is the first row of largest |a| at or
    below j, the rows are swapped across the whole matrix, the column below the diagonal is scaled by the
    reciprocal pivot and the trailing block takes the rank-1 update.  Returns the packed factors (L unit lower
    below the diagonal, U on and above it) and ipiv (1-based pivot rows, as A.ipiv()).  pivot=False: no
    interchanges."""
    A = np.array(A, F64, order="F")
    m, n = A.shape
    mn = min(m, n)
    ipiv = np.arange(1, mn + 1, dtype=np.int64)
    for j in range(mn):
        if pivot:
            p = j + int(np.argmax(np.abs(A[j:, j])))  # argmax returns the first of equal values
            ipiv[j] = p + 1
            if p != j:
                A[[j, p], :] = A[[p, j], :]
        d = A[j, j]
        if d == 0.0:
            raise ZeroDivisionError(f"zero pivot in column {j + 1}")
        A[j + 1:, j] *= 1.0 / d
        A[j + 1:, j + 1:] -= np.outer(A[j + 1:, j], A[j, j + 1:])
    return A, ipiv


def lu_apply_ipiv(A, ipiv) -> np.ndarray:
    """P A: the row interchanges ipiv (1-based) applied in order, as permute_rows_ipiv (include/darray.h:1202)."""
    B = np.array(A, copy=True)
    for i, p in enumerate(np.asarray(ipiv) - 1):
        if p != i:
            B[[i, p], :] = B[[p, i], :]
    return B


def newton_smw(Z, D, g) -> np.ndarray:
    """s = -(Z Z^T + diag(D))^-1 g by Sherman-Morrison-Woodbury: u solves (I + Z^T D^-1 Z) u = -Z^T D^-1 g,
    then s = -D^-1 (g + Z u)."""
    Dinv = 1.0 / D
    Zt = Z * Dinv[:, None]
    M = np.eye(Z.shape[1]) + Z.T @ Zt
    L = np.linalg.cholesky(M)
    rhs = -(Zt.T @ g)
    import scipy.linalg as sl
    u = sl.cho_solve((L, True), rhs)
    return -Dinv * (g + Z @ u)


def newton_smw_bias(Z, D, g, y) -> tuple[np.ndarray, float]:
    """Newton step of the equality-constrained barrier subproblem (y^T a = 0): the bordered system
    [H y; y^T 0] [s; nu] = [-g; 0] with H = Z Z^T + diag(D), solved by two Woodbury solves against one capacity
    matrix: s_g = -H^-1 g, s_y = -H^-1 y, nu = -(y.s_g)/(y.s_y), s = s_g + nu s_y (so y.s = 0).  Returns s, nu."""
    s_g = newton_smw(Z, D, g)
    s_y = newton_smw(Z, D, np.asarray(y, F64))
    nu = -float(y @ s_g) / float(y @ s_y)
    return s_g + nu * s_y, nu


def primal_value(Z, a, C, y=None, b=0.0) -> float:
    """P(w, b) = 0.5 ||w||^2 + C sum max(0, 1 - (z_i.w + y_i b)) at w = Z^T a (labels are folded into Z); b = 0
    for the reference's dual without bias."""
    w = Z.T @ a
    m = Z @ w
    if y is not None and b != 0.0:
        m = m + np.asarray(y, F64) * b
    return 0.5 * float(w @ w) + C * float(np.sum(np.maximum(0.0, 1.0 - m)))


def initial_point(y, C) -> np.ndarray:
    """Class-balanced strictly feasible start (tests/testsvm.cpp:192-212)."""
    y = np.asarray(y)
    plus = int(np.sum(y == 1))
    minus = int(np.sum(y == -1))
    if plus > minus:
        mval = 0.9 * C
        pval = mval * minus / plus
    else:
        pval = 0.9 * C
        mval = pval * plus / minus
    return np.where(y == 1, pval, mval).astype(F64)


@dataclass
class BarrierResult:
    a: np.ndarray
    f: float
    t: float
    outer: int
    newton: int
    gap_barrier: float         # 2n/t / |f|
    gap_primal_dual: float     # (P(Z^T a, b) + f(a)) / |f|
    status: str
    history: list = field(default_factory=list)
    b: float = 0.0             # bias of the decision function (bias=True), from the last Newton step's multiplier


def max_step(a, s, C, frac=0.99) -> float:
    """Largest tau <= 1 keeping 0 < a + tau s < C, times `frac` (correction 5)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        lo = np.where(s < 0, -a / s, np.inf)
        hi = np.where(s > 0, (C - a) / s, np.inf)
    tmax = float(min(lo.min(initial=np.inf), hi.min(initial=np.inf)))
    return min(1.0, frac * tmax)


def svm_barrier(Z, y, C, t0=1.0, mu=20.0, alpha=0.1, beta=0.5, gap_tol=1e-6, newton_tol=1e-6,
                max_outer=60, max_newton=200, a0=None, bias=False) -> BarrierResult:
    """Barrier method of tests/testsvm.cpp:228-321 (constants t0=1, mu=20, alpha=0.1, beta=0.5; Newton stop
    lambda^2/2 < 1e-6 or slow progress; D-condition stop at 1e18) with corrections 4-6.

    bias=True adds the dual's equality constraint y^T a = 0 (the SVM with a bias term, which the reference
    leaves out and estimates afterwards in include/dbarrier.h:420-442): the class-balanced start already satisfies
    it, each Newton step solves the bordered system of newton_smw_bias so the iterates keep it, and the bias is
    the step's multiplier nu (stationarity g + nu y = 0 gives y_i (g(x_i) + nu) = 1 on the margin)."""
    Z = np.asarray(Z, F64)
    n = Z.shape[0]
    yv = np.asarray(y, F64)
    if bias and (np.all(yv == 1) or np.all(yv != 1)):
        raise ValueError("bias needs both classes")
    a = initial_point(y, C) if a0 is None else np.array(a0, F64)
    b = 0.0
    t = t0
    total_newton = 0
    status = "converged"
    hist = []
    outer = 0
    for outer in range(1, max_outer + 1):
        ni = 0
        while True:
            ni += 1
            total_newton += 1
            w = Z.T @ a
            g = (Z @ w - 1.0) + grad_phi(a, C, t)
            D = hess_phi(a, C, t)
            if D.max() / D.min() > 1e18:
                break
            if bias:
                s, b = newton_smw_bias(Z, D, g, yv)
            else:
                s = newton_smw(Z, D, g)
            lam2 = -float(g @ s)
            lastg = gg(a, Z, C, t)
            tau = max_step(a, s, C)
            gs = float(g @ s)
            while gg(a + tau * s, Z, C, t) > lastg + alpha * tau * gs:
                tau *= beta
                if tau < 1e-20:
                    break
            a = a + tau * s
            newg = gg(a, Z, C, t)
            hist.append((outer, ni, t, lam2, tau, newg))
            if lam2 / 2 < newton_tol:
                break
            if ni > 1 and (lastg - newg) < 1e-9 * abs(newg):
                break
            if ni >= max_newton:
                status = "newton_maxiter"
                break
        fa = f(a, Z)
        if 2 * n / t < gap_tol * abs(fa):
            break
        t *= mu
    else:
        status = "outer_maxiter"
    fa = f(a, Z)
    pd = (primal_value(Z, a, C, yv, b) + fa) / abs(fa)
    return BarrierResult(a=a, f=fa, t=t, outer=outer, newton=total_newton, gap_barrier=2 * n / t / abs(fa),
                         gap_primal_dual=pd, status=status, history=hist, b=b)


def decision(Xtest, X, y, a, gamma, block=2048) -> np.ndarray:
    """sum_i a_i y_i K(x_i, x) for each test point (no bias; labels folded into the dual as in the
    reference, include/dkernel.cu:125)."""
    coef = (np.asarray(a, F64) * np.asarray(y, F64))[:, None]
    return sketch(Xtest, X, None, None, coef, gamma, block)[:, 0]


def writemodel(path, a, C, Z, y, X, gamma, minus, plus, bias=None) -> dict:
    """LIBSVM model text as written by include/dbarrier.h:395-470 (bias estimate restated from there: the first 50
    margin support vectors, each with y_j - sum_i a_i y_j ||z_i||^2, averaged).  `bias`: a bias b from a solve of
    the dual with y^T a = 0 (the extension of the barrier that the reference leaves out), written as rho = -b in
    place of the estimate."""
    n = len(a)
    sv = [i for i in range(n) if a[i] > 1e-6]
    bsv = [i for i in sv if a[i] < C - 1e-6]
    if bias is None:
        nb = min(len(bsv), 50)
        bs = []
        zz = np.einsum("ij,ij->i", Z, Z)
        for j in range(nb):
            jj = bsv[j]
            yj = float(y[jj])
            for ii in sv:
                yj -= a[ii] * y[jj] * zz[ii]
            bs.append(yj)
        b = float(np.mean(bs)) if nb else 0.0
    else:
        b = float(bias)
    lines = ["svm_type c_svc", "kernel_type rbf", "gamma %.7f" % gamma, "nr_class 2", "total_sv %d" % len(sv),
             "rho %f" % (-b), "label %d %d" % (plus, minus), "nr_sv %d %d" % (len(bsv), len(sv) - len(bsv)), "SV"]
    for j in sv:
        # "%7f " per nonzero feature, as the reference prints them (a point without any leaves "alpha ")
        feats = "".join("%d:%7f " % (k + 1, X[j, k]) for k in range(X.shape[1]) if X[j, k] != 0)
        lines.append(("%7f " % (y[j] * a[j])) + feats)
    if path is not None:
        with open(path, "w") as fh:
            fh.write("\n".join(lines) + "\n")
    return {"b": b, "nSV": len(sv), "nBSV": len(bsv), "lines": lines}
