"""ctypes front of the sparse basin's CPU oracle (sparse.c). TEST INFRASTRUCTURE ONLY.

Only the tests and the benchmark's CPU-baseline leg import this module; it restates
project!(::SparseBasin) of the reference (src/sflip.jl:1059-2018, src/fgmres.jl) on the CPU
and is the checker, never the product. Parity with the reference itself is unpinned: the
reference runs on Julia and a Vulkan device, neither of which exists here.

A scene is any object with the fields of ``mpp.sparse_scene.SparseScene`` (numpy arrays).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import lib as _oracle_lib

P = ctypes.c_void_p


class OrsGrid(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_float * 3), ("dx", ctypes.c_float), ("nb", ctypes.c_int32 * 3),
                ("radius", ctypes.c_float), ("floor_z", ctypes.c_float)]


class OrsBasin(ctypes.Structure):
    _fields_ = [("g", OrsGrid), ("slot", P), ("where", P), ("nslots", ctypes.c_int32)] + [
        (n, P) for n in ("tf", "tc", "phif", "phic", "Pf", "Pc", "uf", "uc", "vf", "vc", "wf", "wc",
                         "fuf", "fuc", "fvf", "fvc", "fwf", "fwc")]


class OrsOpts(ctypes.Structure):
    _fields_ = [("tol", ctypes.c_float), ("maxiter", ctypes.c_int32), ("sweeps", ctypes.c_int32),
                ("boost", ctypes.c_float), ("fallback", ctypes.c_int32), ("cg_maxiter", ctypes.c_int32)]


class OrsInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("fgmres_iterations", ctypes.c_int32), ("status", ctypes.c_int32),
                ("rel_residual", ctypes.c_float), ("volume", ctypes.c_float), ("gamma", ctypes.c_float)]


_sig_done = False


def _lib():
    global _sig_done
    L = _oracle_lib()
    if not _sig_done:
        B = ctypes.POINTER(OrsBasin)
        i32, f, d = ctypes.c_int, ctypes.c_float, ctypes.c_double
        sig = {
            "ors_volume": (d, [B]), "ors_levels": (i32, [B]),
            "ors_coefficients": (i32, [B] + [P] * 9),
            "ors_apply": (i32, [B, P, P, P, P]),
            "ors_jacobi": (i32, [B, P, P, P, P, P, P]),
            "ors_vcycle": (i32, [B, P, P, P, P, i32, i32, f]),
            "ors_rhs": (i32, [B, f, P, P]),
            "ors_pressure": (i32, [B, P, P, ctypes.POINTER(OrsOpts), ctypes.POINTER(OrsInfo)]),
            "ors_gradient": (i32, [B]),
            "ors_project": (i32, [B, f, d, d, ctypes.POINTER(OrsOpts), ctypes.POINTER(OrsInfo)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _sig_done = True
    return L


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "arrays must be contiguous"
    return ctypes.c_void_p(a.ctypes.data)


def basin_struct(sc) -> OrsBasin:
    """The oracle's view of a scene (its arrays are used in place and must stay alive)."""
    g = sc.grid
    b = OrsBasin()
    b.g = OrsGrid((ctypes.c_float * 3)(*g.lo), g.dx, (ctypes.c_int32 * 3)(*g.nb), g.radius, g.floor_z)
    b.slot = _p(sc.slot)
    b.where = _p(sc.where)
    b.nslots = sc.nslots
    for n in ("tf", "tc", "phif", "phic", "Pf", "Pc", "uf", "uc", "vf", "vc", "wf", "wc",
              "fuf", "fuc", "fvf", "fvc", "fwf", "fwc"):
        setattr(b, n, _p(getattr(sc, n)))
    return b


def opts(tol=1e-4, maxiter=200, sweeps=1, boost=1.0, fallback=False, cg_maxiter=80) -> OrsOpts:
    return OrsOpts(tol, maxiter, sweeps, boost, 1 if fallback else 0, cg_maxiter)


def _info_dict(info: OrsInfo) -> dict:
    return {"iterations": info.iterations, "fgmres_iterations": info.fgmres_iterations, "status": info.status,
            "rel_residual": info.rel_residual, "volume": info.volume, "gamma": info.gamma}


def volume(sc) -> float:
    return _lib().ors_volume(ctypes.byref(basin_struct(sc)))


def levels(sc) -> int:
    return _lib().ors_levels(ctypes.byref(basin_struct(sc)))


def _nc(sc, axis=0):
    n = list(sc.grid.nb)
    n = [4 * v for v in n]
    if axis:
        n[axis - 1] += 1
    return int(np.prod(n))


def coefficients(sc) -> dict:
    """Level 0's couplings, Dirichlet diagonals and coarse activity (coefficients!)."""
    nff, nf = sc.nslots * 4352, sc.nslots * 4096
    out = {k: np.zeros(nff, np.float32) for k in ("cuf", "cvf", "cwf")}
    out.update(cuc=np.zeros(_nc(sc, 1), np.float32), cvc=np.zeros(_nc(sc, 2), np.float32),
               cwc=np.zeros(_nc(sc, 3), np.float32), dDf=np.zeros(nf, np.float32), dDc=np.zeros(_nc(sc), np.float32),
               actc=np.zeros(_nc(sc), np.uint8))
    r = _lib().ors_coefficients(ctypes.byref(basin_struct(sc)), *(_p(out[k]) for k in (
        "cuf", "cvf", "cwf", "cuc", "cvc", "cwc", "dDf", "dDc", "actc")))
    assert r == 0
    return out


def apply(sc, xf, xc):
    qf, qc = np.zeros(sc.nslots * 4096, np.float32), np.zeros(_nc(sc), np.float32)
    assert _lib().ors_apply(ctypes.byref(basin_struct(sc)), _p(xf), _p(xc), _p(qf), _p(qc)) == 0
    return qf, qc


def jacobi(sc, xf, xc, bf, bc):
    of, oc = np.zeros(sc.nslots * 4096, np.float32), np.zeros(_nc(sc), np.float32)
    assert _lib().ors_jacobi(ctypes.byref(basin_struct(sc)), _p(xf), _p(xc), _p(bf), _p(bc), _p(of), _p(oc)) == 0
    return of, oc


def vcycle(sc, rf, rc, sweeps=1, coarse=40, boost=1.0):
    zf, zc = np.zeros(sc.nslots * 4096, np.float32), np.zeros(_nc(sc), np.float32)
    assert _lib().ors_vcycle(ctypes.byref(basin_struct(sc)), _p(rf), _p(rc), _p(zf), _p(zc), sweeps, coarse,
                             boost) == 0
    return zf, zc


def rhs(sc, gamma):
    bf, bc = np.zeros(sc.nslots * 4096, np.float32), np.zeros(_nc(sc), np.float32)
    assert _lib().ors_rhs(ctypes.byref(basin_struct(sc)), gamma, _p(bf), _p(bc)) == 0
    return bf, bc


def pressure(sc, bf, bc, **kw) -> dict:
    """pressure! on (bf, bc) from the warm start in sc.Pf/sc.Pc (updated in place)."""
    info = OrsInfo()
    o = opts(**kw)
    _lib().ors_pressure(ctypes.byref(basin_struct(sc)), _p(bf), _p(bc), ctypes.byref(o), ctypes.byref(info))
    return _info_dict(info)


def gradient(sc) -> None:
    """The velocity update and valid flags from sc.Pf/sc.Pc, in place."""
    assert _lib().ors_gradient(ctypes.byref(basin_struct(sc))) == 0


def project(sc, volume0, dt=1.0 / 48, recover=0.5, **kw) -> dict:
    """project!(s, dt) in place on the scene's arrays."""
    info = OrsInfo()
    o = opts(**kw)
    _lib().ors_project(ctypes.byref(basin_struct(sc)), volume0, dt, recover, ctypes.byref(o), ctypes.byref(info))
    return _info_dict(info)
