"""ctypes binding of libdarray_b200.so (the C ABI declared in include/darray_b200.h).

The library is the product: there is no CPU fallback.  If the shared object is missing, loading raises
instead of degrading silently.
"""
from __future__ import annotations

import ctypes
import os
import re
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libdarray_b200.so"
HEADER = PKG.parent / "include" / "darray_b200.h"

_c_int, _c_float, _c_double = ctypes.c_int, ctypes.c_float, ctypes.c_double
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64


class BarrierParams(ctypes.Structure):
    _fields_ = [("t0", ctypes.c_double), ("mu", ctypes.c_double), ("alpha", ctypes.c_double),
                ("beta", ctypes.c_double), ("gap_tol", ctypes.c_double), ("newton_tol", ctypes.c_double),
                ("max_outer", ctypes.c_int), ("max_newton", ctypes.c_int), ("precision", ctypes.c_int),
                ("refine_max", ctypes.c_int)]


class SvmReport(ctypes.Structure):
    _fields_ = [("f", ctypes.c_double), ("gap_barrier", ctypes.c_double), ("gap_primal_dual", ctypes.c_double),
                ("t", ctypes.c_double), ("nu", ctypes.c_double), ("outer", ctypes.c_int), ("newton", ctypes.c_int),
                ("status", ctypes.c_int), ("refine", ctypes.c_int), ("fallbacks", ctypes.c_int),
                ("ms_sketch", ctypes.c_double), ("ms_orth", ctypes.c_double),
                ("ms_core", ctypes.c_double), ("ms_barrier", ctypes.c_double), ("ms_total", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}

# name -> (restype, argtypes)
SIGNATURES = {
    "db200_create": (_c_int, [ctypes.POINTER(_vp), _c_int, _vp]),
    "db200_destroy": (_c_int, [_vp]),
    "db200_last_error": (ctypes.c_char_p, [_vp]),
    "db200_synchronize": (_c_int, [_vp]),
    "db200_stream": (_vp, [_vp]),
    "db200_launch_count": (_i64, [_vp]),
    "db200_rbf_sketch": (_c_int, [_vp, _c_int, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _vp, _vp,
                                  _vp, _c_int, _vp, _c_int, _c_float]),
    "db200_rbf_block": (_c_int, [_vp, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _vp, _vp, _vp,
                                 _c_int, _c_float]),
    "db200_profile": (_c_int, [_vp, _c_int]),
    "db200_selftest_wait_timeout": (_c_int, [_vp, _c_int]),
    "db200_profile_read": (_c_int, [_vp, ctypes.POINTER(_c_double), ctypes.POINTER(_i64)]),
    "db200_lra_host": (_c_int, [_vp, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _vp, _c_int, _vp, _c_int, _c_float]),
    "db200_potrf": (_c_int, [_vp, _c_int, _vp, _c_int, _c_int]),
    "db200_cholqr2": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _vp, _c_int]),
    "db200_gemm_tn": (_c_int, [_vp, _c_int, _c_int, _c_int, _c_double, _vp, _c_int, _vp, _c_int, _c_double, _vp,
                               _c_int]),
    "db200_trsm_lutn": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _vp, _c_int]),
    "db200_barrier_defaults": (None, [ctypes.POINTER(BarrierParams)]),
    "db200_svm_barrier": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _vp, _c_double, ctypes.POINTER(BarrierParams),
                                   _vp, ctypes.POINTER(SvmReport)]),
    "db200_lowrank": (_c_int, [_vp, _c_int, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _vp, _c_int, _c_float, _c_int,
                               _vp, _c_int, ctypes.POINTER(SvmReport)]),
    "db200_gram_weighted": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _vp, _vp, _c_int, _c_int]),
    "db200_rbf_sketch_f64": (_c_int, [_vp, _c_int, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _c_int, _vp, _vp, _vp,
                                      _c_int, _vp, _c_int, _c_double]),
    "db200_svm_solve": (_c_int, [_vp, _c_int, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _vp, _c_int, _c_float,
                                 _c_double, ctypes.POINTER(BarrierParams), _vp, _vp, _c_int,
                                 ctypes.POINTER(SvmReport)]),
    "db200_default_context": (_vp, []),
    "db200_release_default_context": (_c_int, []),
    "db200_malloc": (_c_int, [_vp, ctypes.c_size_t, ctypes.POINTER(_vp)]),
    "db200_free": (_c_int, [_vp, _vp]),
    "db200_copy_to_device": (_c_int, [_vp, _vp, _vp, ctypes.c_size_t]),
    "db200_copy_to_host": (_c_int, [_vp, _vp, _vp, ctypes.c_size_t]),
    "db200_gemm": (_c_int, [_vp, ctypes.c_char, ctypes.c_char, _c_int, _c_int, _c_int, _c_double, _vp, _c_int, _vp,
                            _c_int, _c_double, _vp, _c_int]),
    "db200_sgemm": (_c_int, [_vp, ctypes.c_char, ctypes.c_char, _c_int, _c_int, _c_int, _c_float, _vp, _c_int, _vp,
                             _c_int, _c_float, _vp, _c_int]),
    "db200_svd_values": (_c_int, [_vp, _c_int, _vp, _c_int, _vp]),
    "db200_knorm": (_c_int, [_vp, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _vp, _c_int, _c_float,
                             ctypes.POINTER(_c_double)]),
    "db200_woodbury_solve": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _vp, _vp, _vp]),
    "db200_vec_update": (_c_int, [_vp, _c_int, _c_double, _vp, _c_double, _vp, _c_double]),
    "db200_barrier_terms": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _vp, _c_double, _c_double, _vp, _vp, _vp, _vp,
                                     ctypes.POINTER(_c_double)]),
    "db200_rbf_sketch_noalloc": (_c_int, [_vp, _c_int, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _vp,
                                          _vp, _vp, _c_int, _vp, _c_int, _c_float]),
}

STATUS = {
    0: "DB200_OK", -1: "DB200_ERR_INVALID", -2: "DB200_ERR_CUDA", -3: "DB200_ERR_NOT_SPD",
    -4: "DB200_ERR_MAXITER", -5: "DB200_ERR_INFEASIBLE", -6: "DB200_ERR_TIMEOUT", -7: "DB200_ERR_NOMEM",
    -8: "DB200_ERR_UNSUPPORTED", -9: "DB200_ERR_TOO_LARGE",
}
NOALLOC_SCRATCH_BYTES = 32 << 20
POINT_MAJOR, FEATURE_MAJOR = 0, 1

_lib = None


class DB200Error(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def header_functions() -> list[str]:
    """Names of every function declared in include/darray_b200.h."""
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:DB200_API\s+)?(?:int|void|const char\s*\*|void\s*\*|int64_t|db200_context\s*\*)\s*\*?\s*(db200_\w+)\s*\(",
                                 text, flags=re.M)))


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m darray_optimizer_b200.build`")
    lib = ctypes.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class Context:
    """Owns a db200_context on one device; `stream` is a raw cudaStream_t (int) or None."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self.lib = load()
        h = _vp()
        st = self.lib.db200_create(ctypes.byref(h), device, stream)
        if st != 0:
            raise DB200Error(st, f"db200_create(device={device}) failed")
        self.h = h

    def check(self, st: int):
        if st != 0:
            msg = self.lib.db200_last_error(self.h)
            raise DB200Error(st, msg.decode() if msg else "")
        return st

    def sync(self):
        return self.check(self.lib.db200_synchronize(self.h))

    @property
    def stream(self) -> int:
        return self.lib.db200_stream(self.h) or 0

    def launches(self) -> int:
        return int(self.lib.db200_launch_count(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.db200_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -------------------------------------------------------------- thin wrappers (device pointers as ints)
    def rbf_sketch(self, m, n, d, l, Xi, ldxi, Xj, ldxj, layout, yi, yj, Om, ldo, Y, ldy, gamma):
        return self.check(self.lib.db200_rbf_sketch(self.h, m, n, d, l, Xi, ldxi, Xj, ldxj, layout, yi, yj, Om,
                                                    ldo, Y, ldy, gamma))

    def profile(self, enable: bool):
        return self.check(self.lib.db200_profile(self.h, 1 if enable else 0))

    def profile_read(self):
        ms, cnt = _c_double(), _i64()
        self.check(self.lib.db200_profile_read(self.h, ctypes.byref(ms), ctypes.byref(cnt)))
        return ms.value, cnt.value

    def lra_host(self, n, d, k, X, ldx, Y, O, ldo, A, lda, gamma):
        return self.check(self.lib.db200_lra_host(self.h, n, d, k, X, ldx, Y, O, ldo, A, lda, gamma))

    def potrf(self, n, A, lda, nb=64):
        return self.check(self.lib.db200_potrf(self.h, n, A, lda, nb))

    def cholqr2(self, n, l, Y, ldy, R, ldr):
        return self.check(self.lib.db200_cholqr2(self.h, n, l, Y, ldy, R, ldr))

    def gemm_tn(self, k, m, n, alpha, A, lda, B, ldb, beta, C, ldc):
        return self.check(self.lib.db200_gemm_tn(self.h, k, m, n, alpha, A, lda, B, ldb, beta, C, ldc))

    def trsm_lutn(self, m, n, R, ldr, B, ldb):
        return self.check(self.lib.db200_trsm_lutn(self.h, m, n, R, ldr, B, ldb))

    @staticmethod
    def barrier_params(**kw) -> BarrierParams:
        p = BarrierParams()
        load().db200_barrier_defaults(ctypes.byref(p))
        for k, v in kw.items():
            setattr(p, k, v)
        return p

    def svm_barrier(self, n, r, Z, ldz, y, C, a, params=None, allow_maxiter=False):
        rep = SvmReport()
        p = params or self.barrier_params()
        st = self.lib.db200_svm_barrier(self.h, n, r, Z, ldz, y, C, ctypes.byref(p), a, ctypes.byref(rep))
        if not (allow_maxiter and st == -4):
            self.check(st)
        return rep

    def lowrank(self, n, d, l, q, X, ldx, y, Om, ldo, gamma, Z, ldz, precision=0):
        rep = SvmReport()
        self.check(self.lib.db200_lowrank(self.h, n, d, l, q, X, ldx, y, Om, ldo, gamma, precision, Z, ldz,
                                          ctypes.byref(rep)))
        return rep

    def gram_weighted(self, n, r, Z, ldz, w, M, ldm, use_tensor_cores):
        return self.check(self.lib.db200_gram_weighted(self.h, n, r, Z, ldz, w, M, ldm, int(use_tensor_cores)))

    def rbf_sketch_f64(self, m, n, d, l, Xi, ldxi, Xj, ldxj, yi, yj, Om, ldo, Y, ldy, gamma):
        return self.check(self.lib.db200_rbf_sketch_f64(self.h, m, n, d, l, Xi, ldxi, Xj, ldxj, yi, yj, Om, ldo, Y,
                                                        ldy, gamma))

    def svm_solve(self, n, d, l, q, X, ldx, y, Om, ldo, gamma, C, a, Z, ldz, params=None):
        rep = SvmReport()
        p = params or self.barrier_params()
        self.check(self.lib.db200_svm_solve(self.h, n, d, l, q, X, ldx, y, Om, ldo, gamma, C, ctypes.byref(p), a, Z,
                                            ldz, ctypes.byref(rep)))
        return rep

    def gemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
        return self.check(self.lib.db200_gemm(self.h, ta.encode(), tb.encode(), m, n, k, alpha, A, lda, B, ldb, beta,
                                              C, ldc))

    def sgemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
        return self.check(self.lib.db200_sgemm(self.h, ta.encode(), tb.encode(), m, n, k, alpha, A, lda, B, ldb,
                                               beta, C, ldc))

    def svd_values(self, n, A, lda, S):
        return self.check(self.lib.db200_svd_values(self.h, n, A, lda, S))

    def knorm(self, n, d, k, X, ldx, y, Z, ldz, gamma):
        out = (_c_double * 3)()
        self.check(self.lib.db200_knorm(self.h, n, d, k, X, ldx, y, Z, ldz, gamma, out))
        return tuple(out)

    def woodbury_solve(self, n, r, Z, ldz, diag, b, x):
        return self.check(self.lib.db200_woodbury_solve(self.h, n, r, Z, ldz, diag, b, x))

    def barrier_terms(self, n, k, Z, ldz, a, C, t, gradf, gradphi, grad, D):
        fg = (_c_double * 2)()
        self.check(self.lib.db200_barrier_terms(self.h, n, k, Z, ldz, a, C, t, gradf, gradphi, grad, D, fg))
        return fg[0], fg[1]

    def rbf_block(self, m, n, d, Xi, ldxi, Xj, ldxj, layout, yi, yj, K, ldk, gamma):
        return self.check(self.lib.db200_rbf_block(self.h, m, n, d, Xi, ldxi, Xj, ldxj, layout, yi, yj, K, ldk,
                                                   gamma))
