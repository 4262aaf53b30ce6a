"""ctypes binding of libmpp.so (include/mpp.h). Loading fails loudly when the library is
missing: there is no CPU fallback."""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "lib", "libmpp.so")

# Status and error codes (include/mpp.h).
OK, NOT_CONVERGED, NONFINITE, INDEFINITE, BREAKDOWN = 0, 1, 2, 3, 4
ERR_INVALID, ERR_CUDA, ERR_NOMEM = -1, -2, -3
PREC = {"fp32": 0, "mixed": 1, "fp16": 1, "bf16": 2, "fp64": 3}
STATUS_NAMES = {OK: "ok", NOT_CONVERGED: "not_converged", NONFINITE: "nonfinite", INDEFINITE: "indefinite",
                BREAKDOWN: "breakdown"}


class Grid(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_float * 3), ("dx", ctypes.c_float), ("n", ctypes.c_int32 * 3),
                ("radius", ctypes.c_float), ("floor_z", ctypes.c_float), ("levels", ctypes.c_int32)]


class Opts(ctypes.Structure):
    _fields_ = [("tol", ctypes.c_float), ("maxiter", ctypes.c_int32), ("sweeps", ctypes.c_int32),
                ("coarse", ctypes.c_int32), ("precision", ctypes.c_int32), ("graph", ctypes.c_int32),
                ("fallback", ctypes.c_int32), ("restart", ctypes.c_int32), ("fallback_maxiter", ctypes.c_int32),
                ("cg_maxiter_with_fallback", ctypes.c_int32), ("sweeps_coarse", ctypes.c_int32)]


class Result(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("status", ctypes.c_int32), ("fallback_used", ctypes.c_int32),
                ("fallback_iterations", ctypes.c_int32), ("rel_residual", ctypes.c_double),
                ("true_rel_residual", ctypes.c_double), ("bnorm", ctypes.c_double), ("volume", ctypes.c_double),
                ("gamma", ctypes.c_float), ("kernel_launches", ctypes.c_int64)]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["status_name"] = STATUS_NAMES.get(self.status, str(self.status))
        return d


class ProfEntry(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 24), ("level", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("launches", ctypes.c_int64), ("ms", ctypes.c_double), ("bytes", ctypes.c_double),
                ("cells", ctypes.c_int64)]


class BasinArrays(ctypes.Structure):
    _fields_ = [("u", ctypes.c_void_p), ("v", ctypes.c_void_p), ("w", ctypes.c_void_p), ("fu", ctypes.c_void_p),
                ("fv", ctypes.c_void_p), ("fw", ctypes.c_void_p), ("P", ctypes.c_void_p), ("types", ctypes.c_void_p),
                ("phi", ctypes.c_void_p), ("volume0", ctypes.c_float)]


class TuneEntry(ctypes.Structure):
    _fields_ = [("smoother", ctypes.c_int32), ("coarse_smoother", ctypes.c_int32), ("sweeps", ctypes.c_int32),
                ("sweeps_coarse", ctypes.c_int32), ("coarse_sweeps", ctypes.c_int32), ("iterations", ctypes.c_int32),
                ("status", ctypes.c_int32), ("ms", ctypes.c_float)]


SMOOTHERS = {0: "vector", 1: "tma", 2: "column", 3: "async"}


class SparseGrid(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_float * 3), ("dx", ctypes.c_float), ("nb", ctypes.c_int32 * 3),
                ("radius", ctypes.c_float), ("floor_z", ctypes.c_float)]


SPARSE_ARRAYS = ("types_f", "types_c", "phi_f", "phi_c", "P_f", "P_c", "u_f", "u_c", "v_f", "v_c", "w_f", "w_c",
                 "fu_f", "fu_c", "fv_f", "fv_c", "fw_f", "fw_c")


class SparseBasinArrays(ctypes.Structure):
    _fields_ = [("slot", ctypes.c_void_p), ("where", ctypes.c_void_p), ("nslots", ctypes.c_int32)] + [
        (n, ctypes.c_void_p) for n in SPARSE_ARRAYS]


class SparseOpts(ctypes.Structure):
    _fields_ = [("tol", ctypes.c_float), ("maxiter", ctypes.c_int32), ("sweeps", ctypes.c_int32),
                ("boost", ctypes.c_float), ("coarse", ctypes.c_int32), ("fallback", ctypes.c_int32),
                ("graph", ctypes.c_int32), ("cg_maxiter", ctypes.c_int32)]


class SparseResult(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("fgmres_iterations", ctypes.c_int32), ("status", ctypes.c_int32),
                ("rel_residual", ctypes.c_float), ("volume", ctypes.c_float), ("gamma", ctypes.c_float),
                ("kernel_launches", ctypes.c_int64)]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["status_name"] = STATUS_NAMES.get(self.status, str(self.status))
        return d


# workspace arrays of mpp_sparse_read
SP_ARRAYS = {n: i for i, n in enumerate(("cu_f", "cv_f", "cw_f", "cu_c", "cv_c", "cw_c", "dD_f", "dD_c", "act_c",
                                          "c1x", "c1y", "c1z", "dD1", "act1", "c2x", "c2y", "c2z", "dD2"))}

# name -> (restype, argtypes); every symbol include/mpp.h declares.
P, I32, F32, F64, SZ = ctypes.c_void_p, ctypes.c_int32, ctypes.c_float, ctypes.c_double, ctypes.c_size_t
_G, _O, _R = ctypes.POINTER(Grid), ctypes.POINTER(Opts), ctypes.POINTER(Result)
SIGNATURES = {
    "mpp_opts_default": (None, [_O]),
    "mpp_levels_for": (I32, [ctypes.POINTER(ctypes.c_int32)]),
    "mpp_ctx_create": (ctypes.c_int, [ctypes.POINTER(P), _G, _O]),
    "mpp_ctx_destroy": (ctypes.c_int, [P]),
    "mpp_ctx_set_opts": (ctypes.c_int, [P, _O]),
    "mpp_ctx_bytes": (SZ, [P]),
    "mpp_volume": (ctypes.c_int, [P, P, ctypes.POINTER(F64), P]),
    "mpp_volume_noalloc": (ctypes.c_int, [_G, P, ctypes.POINTER(F64), P]),
    "mpp_project": (ctypes.c_int, [P, P, P, P, P, P, P, P, P, P, F32, F64, F64, _R, P]),
    "mpp_pressure": (ctypes.c_int, [P, P, P, P, P, _R, P]),
    "mpp_project_vjp": (ctypes.c_int, [P, P, P, P, P, P, P, P, P, P, _R, P]),
    "mpp_vjp_rhs": (ctypes.c_int, [P, P, P, P, P, P, P, P]),
    "mpp_advect": (ctypes.c_int, [P, P, P, P, P, P, P, F32, P]),
    "mpp_batch_create": (ctypes.c_int, [ctypes.POINTER(P), ctypes.c_int, _G, _O]),
    "mpp_batch_destroy": (ctypes.c_int, [P]),
    "mpp_batch_size": (ctypes.c_int, [P]),
    "mpp_batch_set_grouped": (ctypes.c_int, [P, ctypes.c_int]),
    "mpp_batch_groups": (ctypes.c_int, [P]),
    "mpp_batch_ctx": (P, [P, ctypes.c_int]),
    "mpp_batch_project": (ctypes.c_int, [P, ctypes.POINTER(BasinArrays), F64, F64, _R, P]),
    "mpp_ctx_set_smoother": (ctypes.c_int, [P, ctypes.c_int]),
    "mpp_ctx_set_smoothers": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int]),
    "mpp_ctx_smoothers": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "mpp_autotune": (ctypes.c_int, [P, P, P, P, P, P, ctypes.POINTER(TuneEntry), ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_int), P]),
    "mpp_advect_phi": (ctypes.c_int, [P, P, P, P, P, P, F32, P]),
    "mpp_extrapolate": (ctypes.c_int, [P, P, P, P, P, P, P, ctypes.c_int, P]),
    "mpp_redistance": (ctypes.c_int, [P, P, P, ctypes.c_int, P, P]),
    "mpp_classify": (ctypes.c_int, [P, P, P, P]),
    "mpp_filltrapped": (ctypes.c_int, [P, P, P, ctypes.c_int, ctypes.POINTER(ctypes.c_int), P]),
    "mpp_advect_vjp": (ctypes.c_int, [P, P, P, P, P, P, P, F32, P, P, P, P]),
    "mpp_vjp_faces": (ctypes.c_int, [P, P, P, P, P, P, P, P, P, P]),
    "mpp_rhs": (ctypes.c_int, [P, P, P, P, P, P, F32, P]),
    "mpp_diag": (ctypes.c_int, [P, P, P, P, P]),
    "mpp_vcycle": (ctypes.c_int, [P, P, P, P, P, P]),
    "mpp_apply": (ctypes.c_int, [P, P, P, P, P, P]),
    "mpp_gradient": (ctypes.c_int, [P, P, P, P, P, P, P, P, P, P, P]),
    "mpp_solution_f64": (ctypes.c_int, [P, P]),
    "mpp_profile_enable": (ctypes.c_int, [P, ctypes.c_int]),
    "mpp_profile_read": (ctypes.c_int, [P, ctypes.c_void_p, ctypes.c_int]),
    "mpp_sparse_opts_default": (None, [ctypes.POINTER(SparseOpts)]),
    "mpp_sparse_dense_levels": (I32, [ctypes.POINTER(ctypes.c_int32)]),
    "mpp_sparse_ctx_create": (ctypes.c_int, [ctypes.POINTER(P), ctypes.POINTER(SparseGrid), I32]),
    "mpp_sparse_ctx_destroy": (ctypes.c_int, [P]),
    "mpp_sparse_ctx_bytes": (SZ, [P]),
    "mpp_sparse_volume": (ctypes.c_int, [P, ctypes.POINTER(SparseBasinArrays), ctypes.POINTER(F64), P]),
    "mpp_sparse_operator": (ctypes.c_int, [P, ctypes.POINTER(SparseBasinArrays), P]),
    "mpp_sparse_apply": (ctypes.c_int, [P, ctypes.POINTER(SparseBasinArrays), P, P, P, P, P]),
    "mpp_sparse_vcycle": (ctypes.c_int, [P, ctypes.POINTER(SparseBasinArrays), P, P, P, P, I32, I32, F32, P]),
    "mpp_sparse_rhs": (ctypes.c_int, [P, ctypes.POINTER(SparseBasinArrays), F32, P, P, P]),
    "mpp_sparse_pressure": (ctypes.c_int, [P, ctypes.POINTER(SparseBasinArrays), P, P, ctypes.POINTER(SparseOpts),
                                           ctypes.POINTER(SparseResult), P]),
    "mpp_sparse_gradient": (ctypes.c_int, [P, ctypes.POINTER(SparseBasinArrays), P]),
    "mpp_sparse_project": (ctypes.c_int, [P, ctypes.POINTER(SparseBasinArrays), F32, F64, F64,
                                          ctypes.POINTER(SparseOpts), ctypes.POINTER(SparseResult), P]),
    "mpp_sparse_read": (ctypes.c_int64, [P, I32, P, SZ, P]),
    "mpp_last_error": (ctypes.c_char_p, []),
    "mpp_version": (ctypes.c_char_p, []),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libmpp.so and bind every entry point; raises if the library is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libmpp.so is not built ({path}); run maelstrom.jl_b200/build.py")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return load().mpp_last_error().decode(errors="replace")


class MppError(RuntimeError):
    pass


def check(code: int) -> int:
    """Raise on an API/CUDA error (< 0); pass solver statuses (>= 0) through."""
    if code < 0:
        raise MppError(f"libmpp error {code}: {last_error()}")
    return code
