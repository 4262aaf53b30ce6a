"""Many independent basins: one graph launch per batched projection, the autotuner, and
the partition of a batch over GPUs.

:class:`Batch` owns an ``mpp_batch`` (one solver context per basin) and each basin's
arrays on the device; :meth:`Batch.project` is ``project!`` of every basin as one CUDA
graph launch, basins of one size and settings grouped so each pass of their CG loops is one
launch over the group. :meth:`Batch.autotune` times each distinct basin size's own solve over the
smoother forms and sweep counts (``mpp_autotune``) and applies the winner to every basin
of that size. :func:`lpt_partition` splits a batch over ranks (longest processing time
first on cells x expected iterations): basins are independent, so ranks exchange
nothing during the solves. :func:`project_partitioned` is that multi-rank runner: each
rank solves its share (one batched graph launch on its own GPU) and only the per-basin
results are gathered.
"""
from __future__ import annotations

import ctypes
import dataclasses
import heapq

import numpy as np

from . import _lib, grid_struct, scene
from ._lib import check


def lpt_partition(costs, nranks: int) -> list:
    """Greedy LPT: basins in decreasing cost, each to the least loaded rank. Returns one
    list of basin indices per rank (each list in increasing index order)."""
    heap = [(0.0, r) for r in range(nranks)]
    parts = [[] for _ in range(nranks)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def basin_cost(b: "scene.Basin") -> float:
    """Expected solve cost: liquid cells x (levels + 4), a proxy for the iterations of a
    multigrid-preconditioned solve of that size."""
    liquid = float(np.count_nonzero(b.types == scene.LIQUID))
    return liquid * (b.grid.levels + 4)


class Batch:
    def __init__(self, basins: list, device="cuda", *, tol=1e-6, maxiter=100, sweeps=2, coarse=40, precision="fp32",
                 fallback=False):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("libmpp needs a CUDA device")
        self.lib = _lib.load()
        self.basins = basins
        dev = torch.device(device)
        n = len(basins)
        grids = (_lib.Grid * n)(*(grid_struct(b.grid) for b in basins))
        opts = (_lib.Opts * n)()
        for o in opts:
            self.lib.mpp_opts_default(ctypes.byref(o))
            o.tol, o.maxiter, o.sweeps, o.coarse = tol, maxiter, sweeps, coarse
            o.precision, o.graph, o.fallback = _lib.PREC[precision], 1, int(fallback)
        self._opts = dict(tol=tol, maxiter=maxiter, coarse=coarse, precision=_lib.PREC[precision],
                          fallback=int(fallback))
        self._b = ctypes.c_void_p()
        check(self.lib.mpp_batch_create(ctypes.byref(self._b), n, grids, opts))
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self.arrays = []
        for b in basins:
            self.arrays.append(dict(u=t(b.u), v=t(b.v), w=t(b.w), fu=torch.zeros(b.u.size, dtype=torch.uint8, device=dev),
                                    fv=torch.zeros(b.v.size, dtype=torch.uint8, device=dev),
                                    fw=torch.zeros(b.w.size, dtype=torch.uint8, device=dev),
                                    P=torch.zeros(b.grid.ncells, dtype=torch.float32, device=dev), types=t(b.types),
                                    phi=t(b.phi)))
        self.volume0 = []
        for i, a in enumerate(self.arrays):
            vol = ctypes.c_double()
            check(self.lib.mpp_volume(self.ctx(i), ctypes.c_void_p(a["phi"].data_ptr()), ctypes.byref(vol),
                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
            self.volume0.append(vol.value)
        self._structs = None
        self.iterations = []
        self.max_group = 16
        self.grouping = None  # the autotuner's grouping choice and timings

    def ctx(self, i: int) -> ctypes.c_void_p:
        return ctypes.c_void_p(self.lib.mpp_batch_ctx(self._b, i))

    def set_grouped(self, max_group=16):
        """Run basins of one size and settings in groups of at most ``max_group`` (one launch a
        pass for the group; True: 16, the default) or, with ``max_group`` < 2 or False, each
        basin as its own chain (``mpp_batch_set_grouped``)."""
        n = 16 if max_group is True else (0 if max_group is False else int(max_group))
        check(self.lib.mpp_batch_set_grouped(self._b, n))
        self.max_group = n

    @property
    def groups(self) -> int:
        """Groups in the last recorded batch graph."""
        return int(self.lib.mpp_batch_groups(self._b))

    def close(self):
        if getattr(self, "_b", None) and self._b.value:
            self.lib.mpp_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _arrays(self):
        n = len(self.arrays)
        arr = (_lib.BasinArrays * n)()
        for i, a in enumerate(self.arrays):
            arr[i] = _lib.BasinArrays(*(ctypes.c_void_p(a[k].data_ptr()) for k in
                                        ("u", "v", "w", "fu", "fv", "fw", "P", "types", "phi")),
                                      float(self.volume0[i]))
        return arr

    def project(self, dt, recover=0.5, stream=None) -> list:
        """``project!`` of every basin in one graph launch; returns the per-basin results."""
        import torch

        if self._structs is None:
            self._structs = self._arrays()
        n = len(self.arrays)
        res = (_lib.Result * n)()
        s = stream if stream is not None else torch.cuda.current_stream()
        check(self.lib.mpp_batch_project(self._b, self._structs, float(dt), float(recover), res,
                                         ctypes.c_void_p(s.cuda_stream)))
        out = [r for r in res]
        self.iterations.append([r.iterations + r.fallback_iterations for r in out])
        return out

    def autotune(self, stream=None, refine: int = 8) -> dict:
        """Tune each distinct basin size on its first basin (``mpp_autotune``: the basin's
        solve timed alone), then, size by size, time the ``refine`` fastest candidates with the
        whole batch in flight and keep the fastest there: alone, a basin's solve rewards extra
        smoothing that costs throughput when every basin runs at once. The batch's arrays are
        put back after each trial. Returns {dims: {"chosen": (smoother, coarse_smoother,
        sweeps, sweeps_coarse, coarse_sweeps), "table": [...], "batch_ms": {...}}}."""
        import torch

        s = stream if stream is not None else torch.cuda.current_stream()
        groups = {}
        for i, b in enumerate(self.basins):
            groups.setdefault(tuple(b.grid.n), []).append(i)
        report = {}
        for dims, members in groups.items():
            i0 = members[0]
            a = self.arrays[i0]
            table = (_lib.TuneEntry * 128)()
            chosen = ctypes.c_int(-1)
            ptr = lambda k: ctypes.c_void_p(a[k].data_ptr())
            n = check(self.lib.mpp_autotune(self.ctx(i0), ptr("u"), ptr("v"), ptr("w"), ptr("types"), ptr("phi"),
                                            table, 128, ctypes.byref(chosen), ctypes.c_void_p(s.cuda_stream)))
            rows = [dict(smoother=_lib.SMOOTHERS[t.smoother], coarse_smoother=_lib.SMOOTHERS[t.coarse_smoother],
                         sweeps=t.sweeps, sweeps_coarse=t.sweeps_coarse, coarse_sweeps=t.coarse_sweeps, iterations=t.iterations, status=t.status,
                         ms=t.ms) for t in table[:n]]
            if chosen.value >= 0:
                win = table[chosen.value]
                for j in members[1:]:
                    c = self.ctx(j)
                    self._set_sweeps(c, win.sweeps, win.sweeps_coarse, win.coarse_sweeps)
                    check(self.lib.mpp_ctx_set_smoothers(c, win.smoother, win.coarse_smoother))
                report[dims] = dict(chosen=(_lib.SMOOTHERS[win.smoother], _lib.SMOOTHERS[win.coarse_smoother],
                                            win.sweeps, win.sweeps_coarse, win.coarse_sweeps), table=rows)
            else:
                report[dims] = dict(chosen=None, table=rows)
        self._structs = None
        if refine > 1:
            self._refine(groups, report, refine, s)
            self._choose_grouping(report, s)
        return report

    def _choose_grouping(self, report, stream, options=(0, 4, 8, 16)):
        """Time the batch with its basins as chains and in groups of 4, 8 and 16, keep the
        fastest (recorded in self.grouping)."""
        import time

        import torch

        saved = [{n: a[n].clone() for n in ("u", "v", "w", "P")} for a in self.arrays]
        hist = len(self.iterations)
        times = {}
        for g in options:
            self.set_grouped(g)
            best = float("inf")
            for rep in range(3):  # the first launch captures the batch's graph
                for a, sv in zip(self.arrays, saved):
                    for n, t in sv.items():
                        a[n].copy_(t)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                res = self.project(1 / 48, stream=stream)
                torch.cuda.synchronize()
                if any(r.status != 0 for r in res):
                    best = float("inf")
                    break
                if rep:
                    best = min(best, time.perf_counter() - t0)
            times[g] = best
        choice = min(times, key=times.get)
        self.set_grouped(choice)
        self.grouping = {"chosen": choice, "batch_ms": {str(k): round(1e3 * v, 3) for k, v in times.items()}}
        for a, sv in zip(self.arrays, saved):
            for n, t in sv.items():
                a[n].copy_(t)
        del self.iterations[hist:]
        torch.cuda.synchronize()

    def _apply(self, members, cfg):
        fine, coarse, sw, swc, csw = cfg
        for j in members:
            c = self.ctx(j)
            self._set_sweeps(c, sw, swc, csw)
            form = {name: code for code, name in _lib.SMOOTHERS.items()}
            check(self.lib.mpp_ctx_set_smoothers(c, form[fine], form[coarse]))

    def _refine(self, groups, report, k, stream):
        import time

        import torch

        saved = [{n: a[n].clone() for n in ("u", "v", "w", "P")} for a in self.arrays]
        hist = len(self.iterations)

        def batch_seconds():
            best = float("inf")
            for rep in range(3):  # the first launch captures the batch's graph
                for a, sv in zip(self.arrays, saved):
                    for n, t in sv.items():
                        a[n].copy_(t)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                res = self.project(1 / 48, stream=stream)
                torch.cuda.synchronize()
                if any(r.status != 0 for r in res):
                    return float("inf")
                if rep:
                    best = min(best, time.perf_counter() - t0)
            return best

        for dims, members in groups.items():
            rep = report[dims]
            if rep["chosen"] is None:
                continue
            cands = []
            for r in sorted((r for r in rep["table"] if r["status"] == 0), key=lambda r: r["ms"]):
                cfg = (r["smoother"], r["coarse_smoother"], r["sweeps"], r["sweeps_coarse"], r["coarse_sweeps"])
                if cfg not in cands:
                    cands.append(cfg)
                if len(cands) == k:
                    break
            timed = {}
            for cfg in cands:
                self._apply(members, cfg)
                timed[cfg] = batch_seconds()
            best = min(timed, key=timed.get)
            self._apply(members, best)
            rep["chosen"] = best
            rep["batch_ms"] = {",".join(map(str, c)): round(1e3 * t, 3) for c, t in timed.items()}
        for a, sv in zip(self.arrays, saved):
            for n, t in sv.items():
                a[n].copy_(t)
        del self.iterations[hist:]
        torch.cuda.synchronize()

    def _set_sweeps(self, c, sweeps, sweeps_coarse, coarse):
        # the batch's options are the ones it was created with; only the sweeps change
        o = _lib.Opts()
        self.lib.mpp_opts_default(ctypes.byref(o))
        k = self._opts
        o.tol, o.maxiter, o.sweeps, o.coarse = k["tol"], k["maxiter"], sweeps, coarse
        o.sweeps_coarse = sweeps_coarse
        o.precision, o.graph, o.fallback = k["precision"], 1, k["fallback"]
        check(self.lib.mpp_ctx_set_opts(c, ctypes.byref(o)))


@dataclasses.dataclass
class BasinOutcome:
    """One basin's result, as gathered from the rank that solved it."""

    index: int
    rank: int
    iterations: int
    status: int
    true_rel_residual: float
    fallback_used: int = 0


def solve_with_batch(basins, indices, *, dt, tol, maxiter, precision="fp32", autotune=True, steps=1,
                     timer=None):
    """The per-rank solve on this process's GPU: the share's basins in one :class:`Batch`
    (autotuned per size), ``steps`` batched projections (the last one's results returned).
    ``timer(fn)`` may time the projections (it gets a callable that runs them)."""
    share = [basins[i] for i in indices]
    if not share:
        if timer is not None:
            timer(lambda: None)  # the timed region is collective: an idle rank takes part
        return []
    batch = Batch(share, tol=tol, maxiter=maxiter, precision=precision)
    if autotune:
        batch.autotune()
    init = [{k: a[k].clone() for k in ("u", "v", "w")} for a in batch.arrays]
    last = []

    def run():
        nonlocal last
        for _ in range(steps):
            for a, i0 in zip(batch.arrays, init):
                for k in ("u", "v", "w"):
                    a[k].copy_(i0[k])
                a["P"].zero_()
            last = batch.project(dt)

    run()  # the graph's capture and a warm-up
    if timer is not None:
        timer(run)
    else:
        run()
    return [dict(iterations=r.iterations + r.fallback_iterations, status=r.status,
                 true_rel_residual=r.true_rel_residual, fallback_used=r.fallback_used) for r in last]


def project_partitioned(basins, rank: int, world: int, *, solve=None, gather=None, **solve_kw) -> list:
    """Project a batch spread over ``world`` ranks: the basins are split by
    :func:`lpt_partition` on :func:`basin_cost`, this rank solves its share with ``solve``
    (default :func:`solve_with_batch`: one batched graph launch on this rank's GPU), and the
    per-basin results are gathered to every rank (``gather``: default
    ``torch.distributed.all_gather_object``; basins are independent, so nothing else
    crosses ranks). Returns the :class:`BasinOutcome` of every basin, in basin order."""
    parts = lpt_partition([basin_cost(b) for b in basins], world)
    mine = parts[rank]
    solve = solve or solve_with_batch
    local = solve(basins, mine, **solve_kw)
    if len(local) != len(mine):
        raise RuntimeError(f"rank {rank} solved {len(local)} of its {len(mine)} basins")
    payload = [(i, rank, r) for i, r in zip(mine, local)]
    if world > 1:
        if gather is None:
            import torch.distributed as dist

            gathered = [None] * world
            dist.all_gather_object(gathered, payload)
        else:
            gathered = gather(payload)
    else:
        gathered = [payload]
    out = [None] * len(basins)
    for part in gathered:
        for i, r_, res in part:
            if out[i] is not None:
                raise RuntimeError(f"basin {i} solved twice")
            out[i] = BasinOutcome(index=i, rank=r_, **res)
    missing = [i for i, o in enumerate(out) if o is None]
    if missing:
        raise RuntimeError(f"basins {missing} were not solved")
    return out
