"""ctypes front of the CPU oracle (oracle.c). TEST INFRASTRUCTURE ONLY.

Only the tests, the smoke check and the benchmark's CPU-baseline leg import this
module; it is the checker, never the product. It restates src/flip.jl:809-1156 of
the reference on the CPU (see oracle.h); parity with the reference itself is
unpinned because the reference (Julia on Vulkan) cannot run here.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


class Grid(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_float * 3), ("dx", ctypes.c_float), ("n", ctypes.c_int32 * 3),
                ("radius", ctypes.c_float), ("floor_z", ctypes.c_float), ("levels", ctypes.c_int32)]


class Info(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("converged", ctypes.c_int32), ("rnorm", ctypes.c_double),
                ("bnorm", ctypes.c_double), ("volume", ctypes.c_double), ("gamma", ctypes.c_float)]


def build() -> str:
    """Compile liboracle.so with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        G = ctypes.POINTER(Grid)
        I = ctypes.POINTER(Info)
        f, d, i32 = ctypes.c_float, ctypes.c_double, ctypes.c_int
        sig = {
            "orc_volume_f32": (d, [G, P]), "orc_volume_f64": (d, [G, P]),
            "orc_rhs_f32": (None, [G, P, P, P, P, P, f]), "orc_rhs_f64": (None, [G, P, P, P, P, P, d]),
            "orc_diag_f32": (None, [G, P, P, P]), "orc_diag_f64": (None, [G, P, P, P]),
            "orc_coarsen": (None, [P, P, P]),
            "orc_vcycle_f32": (None, [G, P, P, P, P, i32, i32]),
            "orc_vcycle_f64": (None, [G, P, P, P, P, i32, i32]),
            "orc_apply_f32": (None, [G, P, P, P, P]), "orc_apply_f64": (None, [G, P, P, P, P]),
            "orc_gradient_f32": (None, [G, P, P, P, P, P, P, P, P, P]),
            "orc_gradient_f64": (None, [G, P, P, P, P, P, P, P, P, P]),
            "orc_pressure_f32": (i32, [G, P, P, P, P, f, i32, i32, i32, I]),
            "orc_pressure_f64": (i32, [G, P, P, P, P, d, i32, i32, i32, I]),
            "orc_project_f32": (i32, [G, P, P, P, P, P, P, P, P, P, f, d, d, f, i32, i32, i32, I]),
            "orc_project_f64": (i32, [G, P, P, P, P, P, P, P, P, P, d, d, d, d, i32, i32, i32, I]),
            "orc_vjp_rhs_f32": (None, [G, P, P, P, P, P, P]), "orc_vjp_rhs_f64": (None, [G, P, P, P, P, P, P]),
            "orc_vjp_faces_f32": (None, [G, P, P, P, P, P, P, P, P]),
            "orc_vjp_faces_f64": (None, [G, P, P, P, P, P, P, P, P]),
            "orc_project_vjp_f32": (i32, [G, P, P, P, P, P, P, f, i32, i32, i32, I]),
            "orc_project_vjp_f64": (i32, [G, P, P, P, P, P, P, d, i32, i32, i32, I]),
            "orc_advect_f32": (None, [G, P, P, P, P, P, P, P, f]),
            "orc_advect_f64": (None, [G, P, P, P, P, P, P, P, d]),
            "orc_advect_vjp_f32": (None, [G, P, P, P, P, P, P, P, f, P, P, P, P]),
            "orc_advect_vjp_f64": (None, [G, P, P, P, P, P, P, P, d, P, P, P, P]),
            "orc_extrapolate": (None, [G, P, P, P, P, P, P, i32]),
            "orc_redistance": (None, [G, P, i32]), "orc_classify": (None, [G, P, P]),
            "orc_filltrapped": (i32, [G, P, P, i32]),
            "orc_num_threads": (i32, []), "orc_set_num_threads": (None, [i32]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def _grid(g) -> Grid:
    return Grid((ctypes.c_float * 3)(*g.lo), g.dx, (ctypes.c_int32 * 3)(*g.n), g.radius, g.floor, g.levels)


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.c_void_p)


def _ft(prec):
    return np.float32 if prec == 32 else np.float64


def volume(grid, phi, prec=32) -> float:
    phi = np.ascontiguousarray(phi, dtype=_ft(prec))
    return \
        getattr(lib(), f"orc_volume_f{prec}")(ctypes.byref(_grid(grid)), _p(phi))


def rhs(grid, u, v, w, types, gamma, prec=32):
    t = _ft(prec)
    b = np.zeros(grid.ncells, dtype=t)
    u, v, w = (np.ascontiguousarray(a, dtype=t) for a in (u, v, w))
    getattr(lib(), f"orc_rhs_f{prec}")(ctypes.byref(_grid(grid)), _p(b), _p(u), _p(v), _p(w),
                                       _p(np.ascontiguousarray(types, dtype=np.uint8)), gamma)
    return b


def diag(grid, types, phi, prec=32):
    t = _ft(prec)
    d = np.zeros(grid.ncells, dtype=t)
    getattr(lib(), f"orc_diag_f{prec}")(ctypes.byref(_grid(grid)), _p(d),
                                        _p(np.ascontiguousarray(types, dtype=np.uint8)),
                                        _p(np.ascontiguousarray(phi, dtype=t)))
    return d


def coarsen(nf, tf):
    nf = (ctypes.c_int32 * 3)(*nf)
    tc = np.zeros(len(tf) // 8, dtype=np.uint8)
    lib().orc_coarsen(nf, _p(tc), _p(np.ascontiguousarray(tf, dtype=np.uint8)))
    return tc


def _sweeps(sweeps, sweeps_coarse):
    """The C side's packed sweep counts (ORC_SWEEPS in oracle.h): the fine level's, and the
    coarser levels' when given (0: the same as the fine level's, as the reference)."""
    if not (1 <= sweeps <= 255 and 0 <= sweeps_coarse <= 255):
        raise ValueError("sweep counts must be in 1..255")
    return int(sweeps) | (int(sweeps_coarse) << 8)


def vcycle(grid, r, types, diag_, sweeps=2, coarse=40, prec=32, sweeps_coarse=0):
    t = _ft(prec)
    sweeps = _sweeps(sweeps, sweeps_coarse)
    z = np.zeros(grid.ncells, dtype=t)
    getattr(lib(), f"orc_vcycle_f{prec}")(ctypes.byref(_grid(grid)), _p(z), _p(np.ascontiguousarray(r, dtype=t)),
                                          _p(np.ascontiguousarray(types, dtype=np.uint8)),
                                          _p(np.ascontiguousarray(diag_, dtype=t)), sweeps, coarse)
    return z


def apply(grid, x, types, diag_, prec=32):
    t = _ft(prec)
    y = np.zeros(grid.ncells, dtype=t)
    getattr(lib(), f"orc_apply_f{prec}")(ctypes.byref(_grid(grid)), _p(y), _p(np.ascontiguousarray(x, dtype=t)),
                                         _p(np.ascontiguousarray(types, dtype=np.uint8)),
                                         _p(np.ascontiguousarray(diag_, dtype=t)))
    return y


def pressure(grid, P, b, types, phi, tol=1e-4, maxiter=60, sweeps=2, coarse=40, prec=32, sweeps_coarse=0):
    """pressure! on copies: returns (P, info)."""
    t = _ft(prec)
    sweeps = _sweeps(sweeps, sweeps_coarse)
    P = np.array(P, dtype=t, copy=True)
    info = Info()
    getattr(lib(), f"orc_pressure_f{prec}")(ctypes.byref(_grid(grid)), _p(P), _p(np.ascontiguousarray(b, dtype=t)),
                                            _p(np.ascontiguousarray(types, dtype=np.uint8)),
                                            _p(np.ascontiguousarray(phi, dtype=t)), tol, maxiter, sweeps, coarse,
                                            ctypes.byref(info))
    return P, info


def gradient(grid, u, v, w, P, types, phi, prec=32):
    t = _ft(prec)
    u, v, w = (np.array(a, dtype=t, copy=True) for a in (u, v, w))
    fu, fv, fw = (np.zeros(a.size, dtype=np.uint8) for a in (u, v, w))
    getattr(lib(), f"orc_gradient_f{prec}")(ctypes.byref(_grid(grid)), _p(u), _p(v), _p(w), _p(fu), _p(fv), _p(fw),
                                            _p(np.ascontiguousarray(P, dtype=t)),
                                            _p(np.ascontiguousarray(types, dtype=np.uint8)),
                                            _p(np.ascontiguousarray(phi, dtype=t)))
    return u, v, w, fu, fv, fw


def project(basin, P=None, *, volume0=None, dt=1.0 / 48, recover=0.5, tol=1e-4, maxiter=60, sweeps=2, coarse=40,
            prec=32, sweeps_coarse=0):
    """project! on copies of a scene.Basin: returns dict(u, v, w, fu, fv, fw, P, info)."""
    g = basin.grid
    sweeps = _sweeps(sweeps, sweeps_coarse)
    t = _ft(prec)
    u, v, w = (np.array(a, dtype=t, copy=True) for a in (basin.u, basin.v, basin.w))
    fu, fv, fw = (np.zeros(a.size, dtype=np.uint8) for a in (u, v, w))
    P = np.zeros(g.ncells, dtype=t) if P is None else np.array(P, dtype=t, copy=True)
    phi = np.ascontiguousarray(basin.phi, dtype=t)
    if volume0 is None:
        volume0 = volume(g, basin.phi)
    info = Info()
    getattr(lib(), f"orc_project_f{prec}")(ctypes.byref(_grid(g)), _p(u), _p(v), _p(w), _p(fu), _p(fv), _p(fw),
                                           _p(P), _p(np.ascontiguousarray(basin.types, dtype=np.uint8)), _p(phi),
                                           volume0, dt, recover, tol, maxiter, sweeps, coarse, ctypes.byref(info))
    return dict(u=u, v=v, w=w, fu=fu, fv=fv, fw=fw, P=P, info=info)


def vjp_rhs(grid, gu, gv, gw, types, phi, prec=32):
    """beta = dx G^T g on LIQUID cells (the adjoint of project_kernel!, src/flip.jl:1113-1130)."""
    t = _ft(prec)
    beta = np.zeros(grid.ncells, dtype=t)
    getattr(lib(), f"orc_vjp_rhs_f{prec}")(ctypes.byref(_grid(grid)), _p(beta),
                                           *(_p(np.ascontiguousarray(a, dtype=t)) for a in (gu, gv, gw)),
                                           _p(np.ascontiguousarray(types, dtype=np.uint8)),
                                           _p(np.ascontiguousarray(phi, dtype=t)))
    return beta


def vjp_faces(grid, gu, gv, gw, mu, types, prec=32):
    """g_in = g + D^T mu (the adjoint of rhs_kernel!'s divergence, src/flip.jl:817-822)."""
    t = _ft(prec)
    outs = [np.zeros(np.size(a), dtype=t) for a in (gu, gv, gw)]
    getattr(lib(), f"orc_vjp_faces_f{prec}")(ctypes.byref(_grid(grid)), *(_p(o) for o in outs),
                                             *(_p(np.ascontiguousarray(a, dtype=t)) for a in (gu, gv, gw)),
                                             _p(np.ascontiguousarray(mu, dtype=t)),
                                             _p(np.ascontiguousarray(types, dtype=np.uint8)))
    return outs


def project_vjp(basin, gu, gv, gw, mu=None, *, tol=1e-4, maxiter=60, sweeps=2, coarse=40, prec=32):
    """The adjoint of project! w.r.t. (u, v, w) at the basin's types and phi: returns
    dict(gu, gv, gw, mu, info) for the output-face cotangent (gu, gv, gw)."""
    g = basin.grid
    t = _ft(prec)
    gu, gv, gw = (np.array(a, dtype=t, copy=True) for a in (gu, gv, gw))
    mu = np.zeros(g.ncells, dtype=t) if mu is None else np.array(mu, dtype=t, copy=True)
    info = Info()
    getattr(lib(), f"orc_project_vjp_f{prec}")(ctypes.byref(_grid(g)), _p(gu), _p(gv), _p(gw), _p(mu),
                                               _p(np.ascontiguousarray(basin.types, dtype=np.uint8)),
                                               _p(np.ascontiguousarray(basin.phi, dtype=t)), tol, maxiter, sweeps,
                                               coarse, ctypes.byref(info))
    return dict(gu=gu, gv=gv, gw=gw, mu=mu, info=info)


UOFF, VOFF, WOFF, COFF = (0.0, 0.5, 0.5), (0.5, 0.0, 0.5), (0.5, 0.5, 0.0), (0.5, 0.5, 0.5)


def _face_dims(grid, axis):
    n = list(grid.n)
    if axis is not None:
        n[axis] += 1
    return np.array(n, dtype=np.int32)


def advect(grid, src, axis, u, v, w, dt, prec=32):
    """advect_kernel! (src/flip.jl:357-369) of one array: a face array (axis 0, 1, 2) or the
    cell-centred level set (axis None)."""
    t = _ft(prec)
    dims = _face_dims(grid, axis)
    off = np.array((UOFF, VOFF, WOFF)[axis] if axis is not None else COFF, dtype=t)
    out = np.zeros(int(np.prod(dims)), dtype=t)
    getattr(lib(), f"orc_advect_f{prec}")(ctypes.byref(_grid(grid)), _p(out), _p(np.ascontiguousarray(src, dtype=t)),
                                          _p(dims), _p(off),
                                          *(_p(np.ascontiguousarray(a, dtype=t)) for a in (u, v, w)), dt)
    return out


def advect_velocity(grid, u, v, w, dt, prec=32):
    """advect! of the three face arrays through themselves (src/flip.jl:495-497)."""
    return [advect(grid, a, axis, u, v, w, dt, prec) for axis, a in enumerate((u, v, w))]


def advect_velocity_vjp(grid, gou, gov, gow, u, v, w, dt, prec=32):
    """The adjoint of advect_velocity: the cotangent of the advected faces in, that of
    (u, v, w) out (through both the sampled arrays and the traced positions)."""
    t = _ft(prec)
    u, v, w = (np.ascontiguousarray(a, dtype=t) for a in (u, v, w))
    gs = [np.zeros(a.size, dtype=t) for a in (u, v, w)]
    for axis, (go, src) in enumerate(zip((gou, gov, gow), (u, v, w))):
        dims = _face_dims(grid, axis)
        off = np.array((UOFF, VOFF, WOFF)[axis], dtype=t)
        getattr(lib(), f"orc_advect_vjp_f{prec}")(ctypes.byref(_grid(grid)), _p(np.ascontiguousarray(go, dtype=t)),
                                                  _p(src), _p(dims), _p(off), _p(u), _p(v), _p(w), dt,
                                                  _p(gs[axis]), _p(gs[0]), _p(gs[1]), _p(gs[2]))
    return gs


def rollout(basin, u, v, w, steps, dt, *, tol=1e-13, maxiter=400, prec=64, volume0=None, recover=0.5):
    """`steps` steps of advect! (velocity) + project! from (u, v, w) on the basin's types and
    phi: returns the list of per-step start velocities (checkpoints) plus the final one."""
    import dataclasses

    g = basin.grid
    vol0 = volume(g, basin.phi) if volume0 is None else volume0
    states = [[np.array(a, dtype=_ft(prec)) for a in (u, v, w)]]
    for _ in range(steps):
        a = advect_velocity(g, *states[-1], dt, prec)
        bb = dataclasses.replace(basin, u=a[0], v=a[1], w=a[2])
        r = project(bb, volume0=vol0, dt=dt, recover=recover, tol=tol, maxiter=maxiter, prec=prec)
        states.append([r["u"], r["v"], r["w"]])
    return states


def rollout_vjp(basin, states, gu, gv, gw, dt, *, tol=1e-13, maxiter=400, prec=64):
    """The reverse pass of `rollout`: the final velocity's cotangent in, the initial one's
    out (projection adjoint, then advection adjoint at each step's checkpoint)."""
    g = basin.grid
    grad = [np.array(a, dtype=_ft(prec)) for a in (gu, gv, gw)]
    for n in reversed(range(len(states) - 1)):
        r = project_vjp(basin, *grad, tol=tol, maxiter=maxiter, prec=prec)
        grad = advect_velocity_vjp(g, r["gu"], r["gv"], r["gw"], *states[n], dt, prec)
    return grad


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(n)


def extrapolate(grid, u, v, w, fu, fv, fw, layers=6):
    """extrapolate!(s; layers) (src/flip.jl:1192-1206) in Float32: returns new (u, v, w, fu,
    fv, fw), the velocity carried ``layers`` faces out from the flagged faces, zero beyond
    and on walled faces; the flags are the reached ones."""
    out = [np.array(a, dtype=np.float32, copy=True).ravel() for a in (u, v, w)]
    fl = [np.array(a, dtype=np.uint8, copy=True).ravel() for a in (fu, fv, fw)]
    for axis in range(3):
        n = int(np.prod(_face_dims(grid, axis)))
        if out[axis].size != n or fl[axis].size != n:
            raise ValueError(f"face array {axis} has {out[axis].size} / {fl[axis].size} elements, not {n}")
    lib().orc_extrapolate(ctypes.byref(_grid(grid)), *(_p(a) for a in out), *(_p(a) for a in fl), int(layers))
    return (*out, *fl)


def redistance(grid, phi, iterations):
    """redistance!(s; iterations) (src/flip.jl:673-680): returns the new phi (Float32)."""
    out = np.array(phi, dtype=np.float32, copy=True).ravel()
    lib().orc_redistance(ctypes.byref(_grid(grid)), _p(out), int(iterations))
    return out


def classify(grid, phi):
    """classify!(s) (src/flip.jl:682-686): the cell classes from phi and the walls."""
    types = np.zeros(grid.ncells, dtype=np.uint8)
    lib().orc_classify(ctypes.byref(_grid(grid)), _p(types), _p(np.ascontiguousarray(phi, dtype=np.float32)))
    return types


def filltrapped(grid, types, phi, maxrounds=32):
    """filltrapped!(s; maxrounds) (src/flip.jl:747-760): returns (types, phi, rounds)."""
    t = np.array(types, dtype=np.uint8, copy=True).ravel()
    f = np.array(phi, dtype=np.float32, copy=True).ravel()
    rounds = lib().orc_filltrapped(ctypes.byref(_grid(grid)), _p(t), _p(f), int(maxrounds))
    return t, f, rounds
