"""The sparse two-resolution basin's pressure projection on B200 (libmpp's mpp_sparse_*).

This mirrors the reference's interface for ``SparseBasin`` (src/sflip.jl):

* :class:`SparseBasin` holds the arrays ``project!`` reads and writes as CUDA tensors in
  the reference's layout: the block table (``slot``, ``where``, ``nslots``), and each
  field's fine pool and coarse grid (``Field.fine`` / ``Field.coarse``);
* :func:`project` is ``project!(s::SparseBasin, dt; recover)`` (src/sflip.jl:1998-2018),
  :func:`pressure` is ``pressure!(s; tol, maxiter, sweeps, boost)`` (:1867-1904) — with
  ``fallback=True``, the dispatch of src/fgmres.jl:96-110 (CG capped at 80 iterations,
  then FGMRES with tol 5e-4 and boost 1.5 by default) — and :func:`volume` is ``volume(s)``;
* the same return values (iteration counts, pushed to ``s.iterations`` by ``project``) and
  error behaviour (a non-converged CG warns "pressure solve did not converge"; nonfinite
  and indefinite solves raise with the reference's message prefixes; an FGMRES that misses
  its tolerance raises "Pressure did not converge").

All compute runs in libmpp.so's CUDA kernels; this module passes device pointers only and
raises if the library is not built or no GPU is present.
"""
from __future__ import annotations

import ctypes
import warnings

import numpy as np

from . import _lib
from ._lib import SparseBasinArrays, SparseOpts, SparseResult, check

BCELLS, BFACES = 4096, 17 * 256


def _stream_ptr(stream):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


class SparseBasin:
    """The part of the reference's ``SparseBasin`` (src/sflip.jl:252-292) ``project!``
    touches, on the GPU, and the library context that works on it."""

    FIELDS = ("tf", "tc", "phif", "phic", "Pf", "Pc", "uf", "uc", "vf", "vc", "wf", "wc",
              "fuf", "fuc", "fvf", "fvc", "fwf", "fwc")

    def __init__(self, grid, slot, where, nslots, arrays: dict, capacity: int | None = None, opts=None):
        self.grid = grid
        self.slot, self.where, self.nslots = slot, where, int(nslots)
        for k in self.FIELDS:
            setattr(self, k, arrays[k])
        self.iterations = []
        self.volume0 = 0.0
        self.capacity = int(capacity if capacity is not None else max(1, self.nslots))
        self.opts = opts or {}
        lib = _lib.load()
        g = _lib.SparseGrid((ctypes.c_float * 3)(*grid.lo), grid.dx, (ctypes.c_int32 * 3)(*grid.nb), grid.radius,
                            grid.floor_z)
        ctx = ctypes.c_void_p()
        check(lib.mpp_sparse_ctx_create(ctypes.byref(ctx), ctypes.byref(g), self.capacity))
        self._ctx = ctx
        self._lib = lib

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx is not None and ctx.value:
            self._lib.mpp_sparse_ctx_destroy(ctx)
            self._ctx = None

    @classmethod
    def from_scene(cls, sc, device="cuda", capacity=None, **opts) -> "SparseBasin":
        """Upload a ``sparse_scene.SparseScene`` (numpy) to the device; volume0 = volume(s)."""
        import torch

        dev = torch.device(device)
        # an empty pool (no fine blocks) still gets one element, so every pointer is valid
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a if a.size else np.zeros(1, a.dtype))).to(dev)
        arrays = {k: t(getattr(sc, k)) for k in cls.FIELDS}
        s = cls(sc.grid, t(sc.slot), t(np.ascontiguousarray(sc.where.reshape(-1))), sc.nslots, arrays,
                capacity=capacity, opts=opts)
        s.volume0 = volume(s)
        return s

    def arrays(self) -> SparseBasinArrays:
        a = SparseBasinArrays()
        a.slot, a.where, a.nslots = _p(self.slot), _p(self.where), self.nslots
        names = dict(types_f="tf", types_c="tc", phi_f="phif", phi_c="phic", P_f="Pf", P_c="Pc", u_f="uf",
                     u_c="uc", v_f="vf", v_c="vc", w_f="wf", w_c="wc", fu_f="fuf", fu_c="fuc", fv_f="fvf",
                     fv_c="fvc", fw_f="fwf", fw_c="fwc")
        for c_name, attr in names.items():
            setattr(a, c_name, _p(getattr(self, attr)))
        return a

    def options(self, **kw) -> SparseOpts:
        o = SparseOpts()
        self._lib.mpp_sparse_opts_default(ctypes.byref(o))
        merged = dict(self.opts)
        merged.update({k: v for k, v in kw.items() if v is not None})
        if merged.get("fallback"):
            # the dispatch's own defaults (src/fgmres.jl:96)
            o.tol, o.boost, o.maxiter = 5e-4, 1.5, 240
        for k, v in merged.items():
            if k in ("tol", "boost"):
                setattr(o, k, float(v))
            elif k in ("maxiter", "sweeps", "coarse", "cg_maxiter"):
                setattr(o, k, int(v))
            elif k in ("fallback", "graph"):
                setattr(o, k, 1 if v else 0)
            else:
                raise ValueError(f"unknown option {k}")
        return o

    @property
    def bytes(self) -> int:
        return int(self._lib.mpp_sparse_ctx_bytes(self._ctx))

    # ---- pass-level calls (tests, callers that split project!) ----
    def operator(self, stream=None):
        """coefficients! + hierarchy! into the context, from the current classes and level set."""
        a = self.arrays()
        check(self._lib.mpp_sparse_operator(self._ctx, ctypes.byref(a), _stream_ptr(stream)))

    def read(self, name: str):
        """A workspace array of the current operator (see _lib.SP_ARRAYS), as a numpy array."""
        which = _lib.SP_ARRAYS[name]
        dt = np.uint8 if name.startswith("act") else np.float32
        size = self._array_bytes(name)
        out = np.zeros(size // np.dtype(dt).itemsize, dtype=dt)
        n = self._lib.mpp_sparse_read(self._ctx, which, out.ctypes.data_as(ctypes.c_void_p), out.nbytes,
                                      _stream_ptr(None))
        check(int(n))
        return out[: n // np.dtype(dt).itemsize]

    def _array_bytes(self, name: str) -> int:
        nc = [4 * b for b in self.grid.nb]
        faces = lambda a: int(np.prod([n + (i == a - 1) for i, n in enumerate(nc)]))
        sizes = {"cu_f": 4 * self.nslots * BFACES, "cv_f": 4 * self.nslots * BFACES, "cw_f": 4 * self.nslots * BFACES,
                 "cu_c": 4 * faces(1), "cv_c": 4 * faces(2), "cw_c": 4 * faces(3), "dD_f": 4 * self.nslots * BCELLS,
                 "dD_c": 4 * int(np.prod(nc)), "act_c": int(np.prod(nc)), "c1x": 4 * self.nslots * 576,
                 "c1y": 4 * self.nslots * 576, "c1z": 4 * self.nslots * 576, "dD1": 4 * self.nslots * 512,
                 "act1": self.nslots * 512, "c2x": 4 * faces(1), "c2y": 4 * faces(2), "c2z": 4 * faces(3),
                 "dD2": 4 * int(np.prod(nc))}
        return sizes[name]

    def apply(self, xf, xc, qf, qc, stream=None):
        a = self.arrays()
        check(self._lib.mpp_sparse_apply(self._ctx, ctypes.byref(a), _p(xf), _p(xc), _p(qf), _p(qc),
                                         _stream_ptr(stream)))

    def vcycle(self, rf, rc, zf, zc, sweeps=1, coarse=40, boost=1.0, stream=None):
        a = self.arrays()
        check(self._lib.mpp_sparse_vcycle(self._ctx, ctypes.byref(a), _p(rf), _p(rc), _p(zf), _p(zc), sweeps, coarse,
                                          boost, _stream_ptr(stream)))

    def rhs(self, gamma, bf, bc, stream=None):
        a = self.arrays()
        check(self._lib.mpp_sparse_rhs(self._ctx, ctypes.byref(a), gamma, _p(bf), _p(bc), _stream_ptr(stream)))

    def gradient(self, stream=None):
        a = self.arrays()
        check(self._lib.mpp_sparse_gradient(self._ctx, ctypes.byref(a), _stream_ptr(stream)))


def _raise_or_warn(res: SparseResult, fallback: bool):
    if res.status == _lib.NOT_CONVERGED and fallback:
        # the fallback's own miss is an error (src/fgmres.jl:90)
        raise RuntimeError(f"Pressure did not converge: {res.rel_residual:.3e} after {res.iterations} iterations")
    if res.status == _lib.NOT_CONVERGED:
        warnings.warn(f"pressure solve did not converge: residual = {res.rel_residual:.3e}, "
                      f"maxiter = {res.iterations}", RuntimeWarning, stacklevel=3)
    elif res.status == _lib.NONFINITE:
        raise RuntimeError("Nonfinite pressure residual")
    elif res.status == _lib.INDEFINITE:
        raise RuntimeError("Pressure CG requires a positive operator and preconditioner")
    elif res.status == _lib.BREAKDOWN:
        raise RuntimeError("Pressure Arnoldi breakdown")


def volume(s: SparseBasin, stream=None) -> float:
    """``volume(s)`` (src/sflip.jl:1990-1996), m^3."""
    a = s.arrays()
    v = ctypes.c_double()
    check(s._lib.mpp_sparse_volume(s._ctx, ctypes.byref(a), ctypes.byref(v), _stream_ptr(stream)))
    return v.value


def project(s: SparseBasin, dt, recover=0.5, stream=None, **opts) -> SparseBasin:
    """``project!(s::SparseBasin, dt; recover = 0.5)`` (src/sflip.jl:1998-2018)."""
    o = s.options(**opts)
    a = s.arrays()
    res = SparseResult()
    check(s._lib.mpp_sparse_project(s._ctx, ctypes.byref(a), s.volume0, dt, recover, ctypes.byref(o),
                                    ctypes.byref(res), _stream_ptr(stream)))
    s.iterations.append(res.iterations)
    s.last = res
    _raise_or_warn(res, bool(o.fallback))
    return s


def pressure(s: SparseBasin, bf, bc, stream=None, **opts) -> int:
    """``pressure!(s; tol = 1e-4, maxiter = 200, sweeps = 1, boost = 1) -> iterations``
    (src/sflip.jl:1867-1904) for the right-hand side (bf, bc), from the warm start in s.P;
    ``fallback=True`` is the dispatch of src/fgmres.jl:96-110."""
    o = s.options(**opts)
    a = s.arrays()
    res = SparseResult()
    check(s._lib.mpp_sparse_pressure(s._ctx, ctypes.byref(a), _p(bf), _p(bc), ctypes.byref(o), ctypes.byref(res),
                                     _stream_ptr(stream)))
    s.last = res
    _raise_or_warn(res, bool(o.fallback))
    return res.iterations
