"""Maelstrom's dense-MAC pressure projection on B200: the host side of libmpp.

This mirrors the reference's interface for the path (src/flip.jl:809-1156):

* :class:`FlipBasin` holds the arrays ``project!`` reads and writes, as CUDA tensors
  with the reference's shapes and bytes (column-major, i fastest, flattened);
* :func:`project` is ``project!(s, dt; recover, sweeps)`` and :func:`pressure` is
  ``pressure!(s; tol, maxiter, sweeps)``: same argument meaning, same return value
  (``pressure`` returns the iteration count and ``project`` pushes it to
  ``s.iterations``), same error behaviour (a non-converged solve warns
  "pressure solve did not converge"; a nonfinite or indefinite one raises with the
  reference's message prefixes);
* :class:`Projector` is the context the work runs in (libmpp's ``mpp_ctx``).

All compute runs in libmpp.so's CUDA kernels; this module only passes device
pointers. It raises if the library is not built or no GPU is present.
"""
from __future__ import annotations

import ctypes
import dataclasses
import warnings

import numpy as np

from . import _lib
from ._lib import MppError, Result, check
from . import scene

__all__ = ["Projector", "FlipBasin", "project", "pressure", "project_vjp", "extrapolate", "redistance", "classify",
           "filltrapped", "MppError", "scene", "load"]


def load():
    return _lib.load()


def _ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _require(t, dtype, n, name):
    import torch

    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous() or t.numel() != n:
        raise ValueError(f"{name} must be contiguous with {n} elements, got {t.numel()}")


def _stream_ptr(stream):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def grid_struct(g) -> _lib.Grid:
    return _lib.Grid((ctypes.c_float * 3)(*g.lo), g.dx, (ctypes.c_int32 * 3)(*g.n), g.radius, g.floor, g.levels)


class Projector:
    """One basin's solver context (``mpp_ctx``): workspace, levels and CUDA graph.

    ``precision`` is "fp32" (the reference's arithmetic), "fp16"/"mixed" or "bf16"
    (V-cycle stored in 16 bits, flexible CG, FP64 reductions and coarsest solve) or
    "fp64" (the FP64 oracle on the GPU). ``graph=True`` runs each call as one CUDA
    graph launch whose CG loop is a device-side WHILE node.
    """

    def __init__(self, grid, *, tol=1e-4, maxiter=60, sweeps=2, coarse=40, precision="fp32", graph=False,
                 fallback=False, restart=8, fallback_maxiter=240, cg_maxiter_with_fallback=80):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("libmpp needs a CUDA device")
        self.lib = _lib.load()
        self.grid = grid
        self.opts = _lib.Opts()
        self.lib.mpp_opts_default(ctypes.byref(self.opts))
        self.set(tol=tol, maxiter=maxiter, sweeps=sweeps, coarse=coarse, graph=graph, fallback=fallback,
                 restart=restart, fallback_maxiter=fallback_maxiter,
                 cg_maxiter_with_fallback=cg_maxiter_with_fallback, _apply=False)
        self.opts.precision = _lib.PREC[precision]
        self.precision = precision
        self._g = grid_struct(grid)
        self._ctx = ctypes.c_void_p()
        check(self.lib.mpp_ctx_create(ctypes.byref(self._ctx), ctypes.byref(self._g), ctypes.byref(self.opts)))

    def set(self, _apply=True, **kw):
        for k, v in kw.items():
            setattr(self.opts, k, int(v) if k != "tol" else float(v))
        if _apply:
            check(self.lib.mpp_ctx_set_opts(self._ctx, ctypes.byref(self.opts)))

    def close(self):
        if getattr(self, "_ctx", None) and self._ctx.value:
            self.lib.mpp_ctx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nbytes(self) -> int:
        return int(self.lib.mpp_ctx_bytes(self._ctx))

    # ---- whole operations ----
    def project(self, u, v, w, fu, fv, fw, P, types, phi, volume0, dt, recover=0.5, stream=None) -> Result:
        import torch

        g = self.grid
        N = g.ncells
        for t, name, axis in ((u, "u", 0), (v, "v", 1), (w, "w", 2)):
            _require(t, torch.float32, int(np.prod(g.face_shape(axis))), name)
        for t, name, axis in ((fu, "fu", 0), (fv, "fv", 1), (fw, "fw", 2)):
            _require(t, torch.uint8, int(np.prod(g.face_shape(axis))), name)
        _require(P, torch.float32, N, "P")
        _require(types, torch.uint8, N, "types")
        _require(phi, torch.float32, N, "phi")
        res = Result()
        check(self.lib.mpp_project(self._ctx, _ptr(u), _ptr(v), _ptr(w), _ptr(fu), _ptr(fv), _ptr(fw), _ptr(P),
                                   _ptr(types), _ptr(phi), float(volume0), float(dt), float(recover),
                                   ctypes.byref(res), _stream_ptr(stream)))
        return res

    def pressure(self, P, b, types, phi, stream=None) -> Result:
        import torch

        N = self.grid.ncells
        _require(P, torch.float32, N, "P")
        _require(b, torch.float32, N, "b")
        _require(types, torch.uint8, N, "types")
        _require(phi, torch.float32, N, "phi")
        res = Result()
        check(self.lib.mpp_pressure(self._ctx, _ptr(P), _ptr(b), _ptr(types), _ptr(phi), ctypes.byref(res),
                                    _stream_ptr(stream)))
        return res

    def project_vjp(self, gu, gv, gw, mu, types, phi, out=None, stream=None) -> Result:
        """The adjoint of :meth:`project` w.r.t. (u, v, w) (``mpp_project_vjp``): the
        cotangent (gu, gv, gw) of the output faces in, the input faces' cotangent out
        (into ``out`` = (ou, ov, ow), default in place); ``mu`` is the adjoint pressure's
        warm start and result."""
        import torch

        g = self.grid
        for t, name, axis in ((gu, "gu", 0), (gv, "gv", 1), (gw, "gw", 2)):
            _require(t, torch.float32, int(np.prod(g.face_shape(axis))), name)
        ou, ov, ow = out if out is not None else (gu, gv, gw)
        for t, name, axis in ((ou, "ou", 0), (ov, "ov", 1), (ow, "ow", 2)):
            _require(t, torch.float32, int(np.prod(g.face_shape(axis))), name)
        _require(mu, torch.float32, g.ncells, "mu")
        _require(types, torch.uint8, g.ncells, "types")
        _require(phi, torch.float32, g.ncells, "phi")
        res = Result()
        check(self.lib.mpp_project_vjp(self._ctx, _ptr(gu), _ptr(gv), _ptr(gw), _ptr(ou), _ptr(ov), _ptr(ow),
                                       _ptr(mu), _ptr(types), _ptr(phi), ctypes.byref(res), _stream_ptr(stream)))
        return res

    def advect(self, u, v, w, dt, out=None, stream=None):
        """advect! of the face velocities through themselves (``mpp_advect``): returns the
        advected (u, v, w), into ``out`` when given (which must not overlap the inputs)."""
        import torch

        g = self.grid
        for t, name, axis in ((u, "u", 0), (v, "v", 1), (w, "w", 2)):
            _require(t, torch.float32, int(np.prod(g.face_shape(axis))), name)
        outs = out if out is not None else [torch.empty_like(a) for a in (u, v, w)]
        check(self.lib.mpp_advect(self._ctx, *(_ptr(o) for o in outs), _ptr(u), _ptr(v), _ptr(w), float(dt),
                                  _stream_ptr(stream)))
        return outs

    def extrapolate(self, u, v, w, fu, fv, fw, layers=4, stream=None):
        """extrapolate! (``mpp_extrapolate``, src/flip.jl:1192-1206) in place: the velocity
        carried ``layers`` faces out from the faces flagged in (fu, fv, fw), zero on the
        faces no layer reached and on walled faces; the flags end as the reached ones."""
        import torch

        g = self.grid
        for t, name, axis in ((u, "u", 0), (v, "v", 1), (w, "w", 2)):
            _require(t, torch.float32, int(np.prod(g.face_shape(axis))), name)
        for t, name, axis in ((fu, "fu", 0), (fv, "fv", 1), (fw, "fw", 2)):
            _require(t, torch.uint8, int(np.prod(g.face_shape(axis))), name)
        check(self.lib.mpp_extrapolate(self._ctx, _ptr(u), _ptr(v), _ptr(w), _ptr(fu), _ptr(fv), _ptr(fw),
                                       int(layers), _stream_ptr(stream)))

    def redistance(self, phi, phi0, iterations, types=None, stream=None):
        """redistance! (``mpp_redistance``, src/flip.jl:673-680): ``iterations`` Jacobi sweeps
        between phi and phi0 (the reference's two level-set arrays); returns the one holding
        the result (phi0 when ``iterations`` is odd). ``types``, when given, gets classify!
        of the result, fused into the last sweep."""
        import torch

        N = self.grid.ncells
        _require(phi, torch.float32, N, "phi")
        _require(phi0, torch.float32, N, "phi0")
        if types is not None:
            _require(types, torch.uint8, N, "types")
        check(self.lib.mpp_redistance(self._ctx, _ptr(phi), _ptr(phi0), int(iterations),
                                      _ptr(types) if types is not None else None, _stream_ptr(stream)))
        return phi0 if int(iterations) % 2 else phi

    def classify(self, types, phi, stream=None):
        """classify! (``mpp_classify``, src/flip.jl:682-686) into ``types``."""
        import torch

        _require(types, torch.uint8, self.grid.ncells, "types")
        _require(phi, torch.float32, self.grid.ncells, "phi")
        check(self.lib.mpp_classify(self._ctx, _ptr(types), _ptr(phi), _stream_ptr(stream)))

    def filltrapped(self, types, phi, maxrounds=32, stream=None, rounds=True):
        """filltrapped! (``mpp_filltrapped``, src/flip.jl:747-760) in place; returns the sweep
        rounds run (which synchronises the stream), or None with ``rounds=False``."""
        import torch

        _require(types, torch.uint8, self.grid.ncells, "types")
        _require(phi, torch.float32, self.grid.ncells, "phi")
        out = ctypes.c_int(-1)
        check(self.lib.mpp_filltrapped(self._ctx, _ptr(types), _ptr(phi), int(maxrounds),
                                       ctypes.byref(out) if rounds else None, _stream_ptr(stream)))
        return out.value if rounds else None

    def advect_phi(self, phi, u, v, w, dt, stream=None):
        import torch

        _require(phi, torch.float32, self.grid.ncells, "phi")
        out = torch.empty_like(phi)
        check(self.lib.mpp_advect_phi(self._ctx, _ptr(out), _ptr(phi), _ptr(u), _ptr(v), _ptr(w), float(dt),
                                      _stream_ptr(stream)))
        return out

    def advect_vjp(self, gu, gv, gw, u, v, w, dt, out=None, stream=None):
        """The adjoint of :meth:`advect` at velocity (u, v, w): the advected faces'
        cotangent in, (u, v, w)'s out (into ``out``, which may be the cotangent itself)."""
        import torch

        outs = out if out is not None else [torch.empty_like(a) for a in (gu, gv, gw)]
        check(self.lib.mpp_advect_vjp(self._ctx, _ptr(gu), _ptr(gv), _ptr(gw), _ptr(u), _ptr(v), _ptr(w), float(dt),
                                      *(_ptr(o) for o in outs), _stream_ptr(stream)))
        return outs

    def vjp_rhs(self, gu, gv, gw, types, phi, stream=None):
        import torch

        beta = torch.empty(self.grid.ncells, dtype=torch.float32, device=gu.device)
        check(self.lib.mpp_vjp_rhs(self._ctx, _ptr(beta), _ptr(gu), _ptr(gv), _ptr(gw), _ptr(types), _ptr(phi),
                                   _stream_ptr(stream)))
        return beta

    def vjp_faces(self, gu, gv, gw, mu, types, stream=None):
        import torch

        outs = [torch.empty_like(a) for a in (gu, gv, gw)]
        check(self.lib.mpp_vjp_faces(self._ctx, *(_ptr(o) for o in outs), _ptr(gu), _ptr(gv), _ptr(gw), _ptr(mu),
                                     _ptr(types), _stream_ptr(stream)))
        return outs

    def volume(self, phi, stream=None) -> float:
        import torch

        _require(phi, torch.float32, self.grid.ncells, "phi")
        out = ctypes.c_double()
        check(self.lib.mpp_volume(self._ctx, _ptr(phi), ctypes.byref(out), _stream_ptr(stream)))
        return out.value

    # ---- single passes ----
    def rhs(self, u, v, w, types, gamma=0.0, stream=None):
        import torch

        b = torch.empty(self.grid.ncells, dtype=torch.float32, device=u.device)
        check(self.lib.mpp_rhs(self._ctx, _ptr(b), _ptr(u), _ptr(v), _ptr(w), _ptr(types), float(gamma),
                               _stream_ptr(stream)))
        return b

    def diag(self, types, phi, stream=None):
        import torch

        d = torch.empty(self.grid.ncells, dtype=torch.float32, device=types.device)
        check(self.lib.mpp_diag(self._ctx, _ptr(d), _ptr(types), _ptr(phi), _stream_ptr(stream)))
        return d

    def vcycle(self, r, types, phi, stream=None):
        import torch

        z = torch.empty(self.grid.ncells, dtype=torch.float32, device=r.device)
        check(self.lib.mpp_vcycle(self._ctx, _ptr(z), _ptr(r), _ptr(types), _ptr(phi), _stream_ptr(stream)))
        return z

    def apply(self, x, types, phi, stream=None):
        import torch

        y = torch.empty(self.grid.ncells, dtype=torch.float32, device=x.device)
        check(self.lib.mpp_apply(self._ctx, _ptr(y), _ptr(x), _ptr(types), _ptr(phi), _stream_ptr(stream)))
        return y

    def gradient(self, u, v, w, fu, fv, fw, P, types, phi, stream=None):
        check(self.lib.mpp_gradient(self._ctx, _ptr(u), _ptr(v), _ptr(w), _ptr(fu), _ptr(fv), _ptr(fw), _ptr(P),
                                    _ptr(types), _ptr(phi), _stream_ptr(stream)))

    def set_smoothers(self, fine: str, coarse: str | None = None):
        """The smoother form of the fine level and of the coarser row-split levels
        ("vector", "tma" or "column"; ``mpp_ctx_set_smoothers``)."""
        forms = {name: code for code, name in _lib.SMOOTHERS.items()}
        check(self.lib.mpp_ctx_set_smoothers(self._ctx, forms[fine], forms[coarse or fine]))

    def smoothers(self) -> tuple:
        f, c = ctypes.c_int(), ctypes.c_int()
        check(self.lib.mpp_ctx_smoothers(self._ctx, ctypes.byref(f), ctypes.byref(c)))
        return _lib.SMOOTHERS[f.value], _lib.SMOOTHERS[c.value]

    def autotune(self, u, v, w, types, phi, stream=None) -> dict:
        """``mpp_autotune`` on this basin's own solve: keeps the fastest smoother forms and
        sweep counts on the context; returns {"chosen": {...}, "table": [...]}."""
        n = 128
        table = (_lib.TuneEntry * n)()
        chosen = ctypes.c_int(-1)
        k = check(self.lib.mpp_autotune(self._ctx, _ptr(u), _ptr(v), _ptr(w), _ptr(types), _ptr(phi), table, n,
                                        ctypes.byref(chosen), _stream_ptr(stream)))
        rows = [dict(smoother=_lib.SMOOTHERS[t.smoother], coarse_smoother=_lib.SMOOTHERS[t.coarse_smoother],
                     sweeps=t.sweeps, sweeps_coarse=t.sweeps_coarse, coarse_sweeps=t.coarse_sweeps, iterations=t.iterations, status=t.status,
                     ms=round(t.ms, 4)) for t in table[:k]]
        best = rows[chosen.value] if chosen.value >= 0 else None
        if best:
            self.opts.sweeps, self.opts.sweeps_coarse = best["sweeps"], best["sweeps_coarse"]
            self.opts.coarse = best["coarse_sweeps"]
        return {"chosen": best, "table": rows}

    # ---- per-kernel timing ----
    def profile(self, on: bool = True):
        """Bracket every kernel with CUDA events (solves then run their loop from the host)."""
        check(self.lib.mpp_profile_enable(self._ctx, 1 if on else 0))

    def profile_read(self) -> list:
        """[{name, level, launches, ms, bytes, cells}] summed since profiling was turned on."""
        n = check(self.lib.mpp_profile_read(self._ctx, None, 0))
        arr = (_lib.ProfEntry * max(n, 1))()
        check(self.lib.mpp_profile_read(self._ctx, ctypes.cast(arr, ctypes.c_void_p), n))
        out = []
        for e in arr[:n]:
            out.append(dict(name=e.name.decode(), level=e.level, launches=e.launches, ms=e.ms, bytes=e.bytes,
                            cells=e.cells))
        return out

    def solution_f64(self) -> np.ndarray:
        out = np.empty(self.grid.ncells, dtype=np.float64)
        check(self.lib.mpp_solution_f64(self._ctx, out.ctypes.data_as(ctypes.c_void_p)))
        return out


@dataclasses.dataclass
class FlipBasin:
    """The part of the reference's ``FlipBasin`` (src/flip.jl:161-224) the projection
    touches, on the GPU: face velocities and valid flags, pressure (kept as the next
    solve's warm start), cell classes, level set, the start volume and the iteration
    log."""

    grid: object
    u: object
    v: object
    w: object
    fu: object
    fv: object
    fw: object
    P: object
    types: object
    phi: object
    volume0: float
    iterations: list
    projector: Projector | None = None
    band: int = 4  # the narrow band's width in cells (FlipBasin(...; band = 4), src/flip.jl:189)
    phi0: object = None  # the level set's second buffer (s.phi0), allocated by redistance

    @classmethod
    def from_scene(cls, basin: "scene.Basin", device="cuda", **projector_kw) -> "FlipBasin":
        import torch

        dev = torch.device(device)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        g = basin.grid
        s = cls(grid=g, u=t(basin.u), v=t(basin.v), w=t(basin.w),
                fu=torch.zeros(basin.u.size, dtype=torch.uint8, device=dev),
                fv=torch.zeros(basin.v.size, dtype=torch.uint8, device=dev),
                fw=torch.zeros(basin.w.size, dtype=torch.uint8, device=dev),
                P=torch.zeros(g.ncells, dtype=torch.float32, device=dev), types=t(basin.types), phi=t(basin.phi),
                volume0=0.0, iterations=[])
        s.projector = Projector(g, **projector_kw)
        s.volume0 = s.projector.volume(s.phi)  # initialize!: s.volume0 = volume(s) (src/flip.jl:346)
        return s


def project_vjp(s: FlipBasin, gu, gv, gw, mu=None):
    """The pullback of ``project!(s, dt)`` w.r.t. (s.u, s.v, s.w) at the basin's current
    types and phi (the rrule's pullback): the output faces' cotangent in, in place, the
    input faces' cotangent out. ``mu`` (adjoint pressure) defaults to a zero start kept
    on the basin for the next call's warm start."""
    import torch

    if mu is None:
        if getattr(s, "mu", None) is None:
            s.mu = torch.zeros(s.grid.ncells, dtype=torch.float32, device=s.P.device)
        mu = s.mu
    res = s.projector.project_vjp(gu, gv, gw, mu, s.types, s.phi)
    s.last_vjp = res
    _raise_or_warn(res)
    return gu, gv, gw


def _raise_or_warn(res: Result, bnorm_ok=True):
    if res.status == _lib.NOT_CONVERGED and res.fallback_used:
        # the fallback's own miss is an error (src/fgmres.jl:90)
        raise RuntimeError(f"Pressure did not converge: {res.true_rel_residual:.3e} after "
                           f"{res.iterations} + {res.fallback_iterations} iterations")
    if res.status == _lib.NOT_CONVERGED:
        warnings.warn(f"pressure solve did not converge: residual = {res.rel_residual:.3e}, "
                      f"iterations = {res.iterations}", RuntimeWarning, stacklevel=3)
    elif res.status == _lib.NONFINITE:
        raise RuntimeError("Nonfinite pressure residual")
    elif res.status == _lib.INDEFINITE:
        raise RuntimeError("Pressure CG requires a positive operator and preconditioner")
    elif res.status == _lib.BREAKDOWN:
        raise RuntimeError("Pressure Arnoldi breakdown")


def project(s: FlipBasin, dt, recover=0.5, sweeps=None) -> FlipBasin:
    """``project!(s, dt; recover = 0.5, sweeps = 2)`` (src/flip.jl:1144-1156)."""
    p = s.projector
    if sweeps is not None and sweeps != p.opts.sweeps:
        p.set(sweeps=sweeps)
    res = p.project(s.u, s.v, s.w, s.fu, s.fv, s.fw, s.P, s.types, s.phi, s.volume0, dt, recover)
    # with the fallback, pressure! counts CG's and FGMRES's iterations (src/fgmres.jl:110)
    s.iterations.append(res.iterations + res.fallback_iterations)
    s.last = res
    _raise_or_warn(res)
    return s


def extrapolate(s: FlipBasin, layers=4) -> FlipBasin:
    """``extrapolate!(s; layers = 4)`` (src/flip.jl:1192-1206); ``step!`` calls it with
    ``layers = 6`` right after ``project!`` (:1403-1404)."""
    s.projector.extrapolate(s.u, s.v, s.w, s.fu, s.fv, s.fw, layers)
    return s


def redistance(s: FlipBasin, iterations=None) -> FlipBasin:
    """``redistance!(s; iterations = s.band + 3)`` (src/flip.jl:673-680): the Jacobi sweeps
    ping-pong between ``s.phi`` and ``s.phi0`` and the two swap as the reference's do, so
    ``s.phi`` holds the result."""
    import torch

    it = s.band + 3 if iterations is None else int(iterations)
    if s.phi0 is None:
        s.phi0 = torch.empty_like(s.phi)
    out = s.projector.redistance(s.phi, s.phi0, it)
    if out is not s.phi:
        s.phi, s.phi0 = s.phi0, s.phi
    return s


def classify(s: FlipBasin) -> FlipBasin:
    """``classify!(s)`` (src/flip.jl:682-686)."""
    s.projector.classify(s.types, s.phi)
    return s


def filltrapped(s: FlipBasin, maxrounds=32) -> FlipBasin:
    """``filltrapped!(s; maxrounds = 32)`` (src/flip.jl:747-760); the rounds it ran are kept
    in ``s.trap_rounds``."""
    s.trap_rounds = s.projector.filltrapped(s.types, s.phi, maxrounds)
    return s


def pressure(s: FlipBasin, b, tol=None, maxiter=None, sweeps=None) -> int:
    """``pressure!(s; tol = 1e-4, maxiter = 60, sweeps = 2) -> iterations``
    (src/flip.jl:1082-1111), for the right-hand side ``b``."""
    p = s.projector
    kw = {k: v for k, v in (("tol", tol), ("maxiter", maxiter), ("sweeps", sweeps)) if v is not None}
    if kw:
        p.set(**kw)
    res = p.pressure(s.P, b, s.types, s.phi)
    s.last = res
    _raise_or_warn(res)
    return res.iterations + res.fallback_iterations
