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
                ("refine_max", ctypes.c_int), ("bias", ctypes.c_int)]


class SvmReport(ctypes.Structure):
    _fields_ = [("f", ctypes.c_double), ("gap_barrier", ctypes.c_double), ("gap_primal_dual", ctypes.c_double),
                ("t", ctypes.c_double), ("nu", ctypes.c_double), ("outer", ctypes.c_int), ("newton", ctypes.c_int),
                ("status", ctypes.c_int), ("refine", ctypes.c_int), ("fallbacks", ctypes.c_int),
                ("ms_sketch", ctypes.c_double), ("ms_orth", ctypes.c_double),
                ("ms_core", ctypes.c_double), ("ms_barrier", ctypes.c_double), ("ms_total", ctypes.c_double),
                ("b", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LandmarkReport(ctypes.Structure):
    _fields_ = [("used_fallback", ctypes.c_int), ("rank", ctypes.c_int), ("residual_est", ctypes.c_double),
                ("residual_fallback", ctypes.c_double), ("ms_features", ctypes.c_double),
                ("ms_predict", ctypes.c_double), ("ms_select", ctypes.c_double), ("ms_factor", ctypes.c_double),
                ("ms_residual", ctypes.c_double), ("ms_fallback", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SketchJob(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int), ("n", ctypes.c_int), ("d", ctypes.c_int), ("l", ctypes.c_int),
                ("Xi", ctypes.c_void_p), ("ldxi", ctypes.c_int), ("Xj", ctypes.c_void_p), ("ldxj", ctypes.c_int),
                ("yi", ctypes.c_void_p), ("yj", ctypes.c_void_p), ("Omega", ctypes.c_void_p), ("ldo", ctypes.c_int),
                ("Y", ctypes.c_void_p), ("ldy", ctypes.c_int), ("gamma", ctypes.c_float),
                ("n_panels", ctypes.c_int), ("panel", ctypes.c_int), ("g_bufs", ctypes.c_int)]


class SvmInstance(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("d", ctypes.c_int), ("l", ctypes.c_int), ("X", ctypes.c_void_p),
                ("ldx", ctypes.c_int), ("y", ctypes.c_void_p), ("gamma", ctypes.c_float), ("C", ctypes.c_double),
                ("Omega", ctypes.c_void_p), ("ldo", ctypes.c_int), ("Z", ctypes.c_void_p), ("ldz", ctypes.c_int),
                ("a", ctypes.c_void_p), ("n_panels", ctypes.c_int), ("panel", ctypes.c_int),
                ("g_bufs", ctypes.c_int)]


class BatchReport(ctypes.Structure):
    _fields_ = [("ms_pack", ctypes.c_double), ("ms_sketch", ctypes.c_double), ("ms_orth", ctypes.c_double),
                ("ms_core", ctypes.c_double), ("ms_barrier", ctypes.c_double), ("ms_total", ctypes.c_double),
                ("kernel_passes", ctypes.c_int), ("graph_replays", ctypes.c_int), ("workers", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_u64 = ctypes.c_uint64
_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)

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
    "db200_rbf_sketch_ex": (_c_int, [_vp, _c_int, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _vp,
                                     _vp, _vp, _c_int, _vp, _c_int, _c_float, _c_int]),
    "db200_rbf_block": (_c_int, [_vp, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _vp, _vp, _vp,
                                 _c_int, _c_float]),
    "db200_profile": (_c_int, [_vp, _c_int]),
    "db200_probe_fp64_peak": (_c_int, [_vp, ctypes.POINTER(_c_double), ctypes.POINTER(_c_double)]),
    "db200_selftest_wait_timeout": (_c_int, [_vp, _c_int]),
    "db200_selftest_grid_barrier_timeout": (_c_int, [_vp, _c_int]),
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
    "db200_rbf_block_f64": (_c_int, [_vp, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _c_int, _vp, _vp, _vp, _c_int,
                                     _c_double]),
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
    # batched instances
    "db200_rbf_sketch_batched": (_c_int, [_vp, _c_int, ctypes.POINTER(SketchJob)]),
    "db200_svm_solve_batched": (_c_int, [_vp, _c_int, ctypes.POINTER(SvmInstance), _c_int,
                                         ctypes.POINTER(BarrierParams), _c_int, _c_int, ctypes.POINTER(SvmReport),
                                         ctypes.POINTER(BatchReport)]),
    # learned landmarks
    "db200_knn_distance": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _c_int, _vp, _c_int, _vp]),
    "db200_leverage_features": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _vp, _vp]),
    "db200_ridge_leverage": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _c_double, _vp]),
    "db200_mlp_create": (_c_int, [_vp, _c_int, _c_int, _c_int, _u64, ctypes.POINTER(_vp)]),
    "db200_mlp_destroy": (None, [_vp]),
    "db200_mlp_param_count": (_c_int, [_vp]),
    "db200_mlp_get_params": (_c_int, [_vp, _vp, _fp]),
    "db200_mlp_set_params": (_c_int, [_vp, _vp, _fp]),
    "db200_mlp_set_input_scaling": (_c_int, [_vp, _vp, _fp, _fp]),
    "db200_mlp_forward": (_c_int, [_vp, _vp, _c_int, _vp, _vp]),
    "db200_mlp_gradients": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _fp, _vp]),
    "db200_mlp_adam_step": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _c_float, _fp]),
    "db200_gumbel_keys": (_c_int, [_vp, _c_int, _vp, _u64, _vp]),
    "db200_select_topk": (_c_int, [_vp, _c_int, _vp, _c_int, _vp]),
    "db200_landmark_factor": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _vp, _c_float, _c_int, _vp, _vp, _c_int,
                                       _dp]),
    "db200_landmark_factor_ex": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _vp, _c_float, _c_int, _vp, _vp, _c_int,
                                          _dp, _c_int]),
    "db200_residual_estimate": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _vp, _c_float, _c_int, _vp, _c_int,
                                         _c_int, _vp, _dp]),
    "db200_select_landmarks": (_c_int, [_vp, _c_int, _c_int, _c_int, _vp, _c_int, _vp, ctypes.c_ulonglong, _c_int,
                                        _vp]),
    "db200_svm_solve_landmarks": (_c_int, [_vp, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _c_float, _c_double, _vp,
                                           _u64, _c_int, _c_int, _c_double, _vp, _c_int, _c_int, _c_int,
                                           ctypes.POINTER(BarrierParams), _vp, _vp, _c_int, ctypes.POINTER(SvmReport),
                                           ctypes.POINTER(LandmarkReport)]),
    "db200_lu_factorize": (_c_int, [_vp, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _c_int, _c_int]),
    "db200_libsvm_parse": (_c_int, [_vp, _vp, ctypes.c_longlong, _c_int, _c_int, _c_int, _vp, ctypes.c_longlong, _vp,
                                    ctypes.POINTER(_c_int)]),
    "db200_read_libsvm": (_c_int, [_vp, ctypes.c_char_p, _c_int, _c_int, _c_int, _vp, ctypes.c_longlong, _vp,
                                   ctypes.POINTER(_c_int)]),
}

# all-reduce callback of a row-sharded solve (include/darray_b200.h: db200_allreduce_fn)
ALLREDUCE_FN = ctypes.CFUNCTYPE(_c_int, _vp, _vp, ctypes.c_longlong, _c_int, _vp)


class Collective(ctypes.Structure):
    _fields_ = [("world", _c_int), ("rank", _c_int), ("allreduce", ALLREDUCE_FN), ("user", _vp)]


SIGNATURES.update({
    "db200_set_collective": (_c_int, [_vp, ctypes.POINTER(Collective)]),
    "db200_row_shard": (_c_int, [_c_int, _c_int, _c_int, ctypes.POINTER(_c_int), ctypes.POINTER(_c_int)]),
})

STATUS = {
    0: "DB200_OK", -1: "DB200_ERR_INVALID", -2: "DB200_ERR_CUDA", -3: "DB200_ERR_NOT_SPD",
    -4: "DB200_ERR_MAXITER", -5: "DB200_ERR_INFEASIBLE", -6: "DB200_ERR_TIMEOUT", -7: "DB200_ERR_NOMEM",
    -8: "DB200_ERR_UNSUPPORTED", -9: "DB200_ERR_TOO_LARGE", -10: "DB200_ERR_SINGULAR",
    -11: "DB200_ERR_COLLECTIVE",
}
REDUCE_SUM, REDUCE_MAX, REDUCE_MIN = 0, 1, 2
NOALLOC_SCRATCH_BYTES = 32 << 20
# precisions of the SVM path and sketch products (include/darray_b200.h)
MIXED, FP64, MIXED_FAST = 0, 1, 2
SKETCH_SINGLE, SKETCH_P_SPLIT, SKETCH_COMPENSATED, SKETCH_COMPENSATED_PROMOTED = 0, 1, 2, 3
SKETCH_COMPENSATED_PROMOTED_COARSE = 4
POINT_MAJOR, FEATURE_MAJOR = 0, 1
F32, F64 = 0, 1

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

    def set_collective(self, world: int, rank: int, fn=None):
        """Attach a row-sharding collective (fn: an ALLREDUCE_FN, kept alive here) or detach (world 1)."""
        self._collective_fn = fn
        if world <= 1 or fn is None:
            return self.check(self.lib.db200_set_collective(self.h, None))
        c = Collective(world, rank, fn, None)
        return self.check(self.lib.db200_set_collective(self.h, ctypes.byref(c)))

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

    def rbf_sketch_ex(self, m, n, d, l, Xi, ldxi, Xj, ldxj, layout, yi, yj, Om, ldo, Y, ldy, gamma, product):
        return self.check(self.lib.db200_rbf_sketch_ex(self.h, m, n, d, l, Xi, ldxi, Xj, ldxj, layout, yi, yj, Om,
                                                       ldo, Y, ldy, gamma, product))

    def probe_fp64_peak(self):
        """(DMMA, DFMA) TFLOP/s measured on this GPU."""
        a, b = _c_double(), _c_double()
        self.check(self.lib.db200_probe_fp64_peak(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

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

    def rbf_block_f64(self, m, n, d, Xi, ldxi, Xj, ldxj, yi, yj, K, ldk, gamma):
        return self.check(self.lib.db200_rbf_block_f64(self.h, m, n, d, Xi, ldxi, Xj, ldxj, yi, yj, K, ldk, gamma))

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

    # ------------------------------------------------------------------ batched instances
    def rbf_sketch_batched(self, jobs):
        arr = (SketchJob * len(jobs))(*jobs)
        return self.check(self.lib.db200_rbf_sketch_batched(self.h, len(jobs), arr))

    def svm_solve_batched(self, instances, q=1, params=None, use_graph=True, workers=8):
        arr = (SvmInstance * len(instances))(*instances)
        reps = (SvmReport * len(instances))()
        brep = BatchReport()
        p = params or self.barrier_params()
        st = self.lib.db200_svm_solve_batched(self.h, len(instances), arr, q, ctypes.byref(p), int(use_graph),
                                              workers, reps, ctypes.byref(brep))
        if st not in (0, -4):
            self.check(st)
        return list(reps), brep

    # ------------------------------------------------------------------ learned landmarks
    def knn_distance(self, n, d, X, ldx, s, ref_idx, k, out):
        return self.check(self.lib.db200_knn_distance(self.h, n, d, X, ldx, s, ref_idx, k, out))

    def leverage_features(self, n, d, X, ldx, knn, F):
        return self.check(self.lib.db200_leverage_features(self.h, n, d, X, ldx, knn, F))

    def ridge_leverage(self, n, r, Z, ldz, lam, lev):
        return self.check(self.lib.db200_ridge_leverage(self.h, n, r, Z, ldz, lam, lev))

    def gumbel_keys(self, n, logits, seed, keys):
        return self.check(self.lib.db200_gumbel_keys(self.h, n, logits, seed, keys))

    def select_topk(self, n, keys, k, idx):
        return self.check(self.lib.db200_select_topk(self.h, n, keys, k, idx))

    def landmark_factor(self, n, d, X, ldx, y, gamma, r, idx, Z, ldz, precision=None):
        nu = _c_double()
        if precision is None:
            self.check(self.lib.db200_landmark_factor(self.h, n, d, X, ldx, y, gamma, r, idx, Z, ldz,
                                                      ctypes.byref(nu)))
        else:
            self.check(self.lib.db200_landmark_factor_ex(self.h, n, d, X, ldx, y, gamma, r, idx, Z, ldz,
                                                         ctypes.byref(nu), precision))
        return nu.value

    def residual_estimate(self, n, d, X, ldx, y, gamma, r, Z, ldz, s, sample_idx):
        est = _c_double()
        self.check(self.lib.db200_residual_estimate(self.h, n, d, X, ldx, y, gamma, r, Z, ldz, s, sample_idx,
                                                    ctypes.byref(est)))
        return est.value

    def select_landmarks(self, n, d, r, X, ldx, net, seed, s_knn, idx):
        return self.check(self.lib.db200_select_landmarks(self.h, n, d, r, X, ldx, net.h, seed, s_knn, idx))

    def svm_solve_landmarks(self, n, d, r, X, ldx, y, gamma, C, net, seed, s_knn, s_res, tol, Omega, ldo, l_fb, q,
                            a, Z, ldz, params=None):
        rep, lrep = SvmReport(), LandmarkReport()
        p = params or self.barrier_params()
        st = self.lib.db200_svm_solve_landmarks(self.h, n, d, r, X, ldx, y, gamma, C, net.h, seed, s_knn, s_res, tol,
                                                Omega, ldo, l_fb, q, ctypes.byref(p), a, Z, ldz, ctypes.byref(rep),
                                                ctypes.byref(lrep))
        if st not in (0, -4):
            self.check(st)
        return rep, lrep

    def lu_factorize(self, m, n, A, lda, ipiv, pivot=1, nleft=0, swap_left_panels=1):
        return self.check(self.lib.db200_lu_factorize(self.h, m, n, nleft, A, lda, ipiv, pivot, swap_left_panels))

    def libsvm_parse(self, text, nbytes, n, d, dtype, X, ldx, y):
        """db200_libsvm_parse on device text; returns the lines parsed."""
        lines = _c_int()
        self.check(self.lib.db200_libsvm_parse(self.h, text, nbytes, n, d, dtype, X, ldx, y, ctypes.byref(lines)))
        return lines.value

    def read_libsvm(self, path, n, d, dtype, X, ldx, y):
        """db200_read_libsvm into host X and y (pointers); returns the lines parsed."""
        lines = _c_int()
        self.check(self.lib.db200_read_libsvm(self.h, str(path).encode(), n, d, dtype, X, ldx, y,
                                              ctypes.byref(lines)))
        return lines.value


class Mlp:
    """The leverage MLP (db200_mlp): `hidden` ReLU layers of `width`, one linear output, on one context."""

    def __init__(self, ctx: Context, in_dim: int, width: int = 256, hidden: int = 3, seed: int = 0):
        self.ctx = ctx
        h = _vp()
        ctx.check(ctx.lib.db200_mlp_create(ctx.h, in_dim, width, hidden, seed, ctypes.byref(h)))
        self.h = h
        self.in_dim, self.width, self.hidden = in_dim, width, hidden

    @property
    def nparams(self) -> int:
        return int(self.ctx.lib.db200_mlp_param_count(self.h))

    def get_params(self):
        import numpy as np
        out = np.empty(self.nparams, dtype=np.float32)
        self.ctx.check(self.ctx.lib.db200_mlp_get_params(self.ctx.h, self.h, out.ctypes.data_as(_fp)))
        return out

    def set_params(self, params):
        import numpy as np
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == self.nparams
        self.ctx.check(self.ctx.lib.db200_mlp_set_params(self.ctx.h, self.h, p.ctypes.data_as(_fp)))

    def set_input_scaling(self, mean, scale):
        import numpy as np
        m = np.ascontiguousarray(mean, dtype=np.float32)
        s = np.ascontiguousarray(scale, dtype=np.float32)
        self.ctx.check(self.ctx.lib.db200_mlp_set_input_scaling(self.ctx.h, self.h, m.ctypes.data_as(_fp),
                                                               s.ctypes.data_as(_fp)))

    def forward(self, m, F, out):
        return self.ctx.check(self.ctx.lib.db200_mlp_forward(self.ctx.h, self.h, m, F, out))

    def gradients(self, m, F, target, grads):
        loss = ctypes.c_float()
        self.ctx.check(self.ctx.lib.db200_mlp_gradients(self.ctx.h, self.h, m, F, target, ctypes.byref(loss), grads))
        return loss.value

    def adam_step(self, m, F, target, lr):
        loss = ctypes.c_float()
        self.ctx.check(self.ctx.lib.db200_mlp_adam_step(self.ctx.h, self.h, m, F, target, lr, ctypes.byref(loss)))
        return loss.value

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.db200_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
