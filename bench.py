#!/usr/bin/env python
"""Benchmark of the dense-MAC pressure projection (Maelstrom.jl's FlipBasin project!).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mpp|reference]

One step = one projection (project!: volume and gamma, rhs, clearair, the pressure
solve to 1e-6 relative residual, the gradient update with valid flags) of the 256^3
basin with a Rankine vortex (Gamma = 225 m^2/s, core 2.5 m), FP32 face velocities
uniform[-1, 1) m/s from seed 1001, synthetic. Each step restores the input velocities
and starts the solve from P = 0, so every step does the same work.

`value` is the mixed-precision (FP16-stored V-cycle, FP32 compute, FP64 reductions and
coarsest solve), graph-captured projection rate; the plain FP32 form's rate is in
`fp32_plain`. `e2e` is the same projection through the public API with the inputs in
pinned host memory: every step copies u, v, w, types, phi, P to the device and reads
u, v, w, fu, fv, fw, P back. Multi-GPU runs are independent replicas (the projection of
one basin does not shard): `value` sums the ranks' rates, timed as the slowest rank.

`--impl reference` times the CPU restatement of the reference's projection (the
oracle; the reference itself is Julia on Vulkan and cannot run here) on the host's
cores, on the same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "maelstrom.jl_b200"))
sys.path.insert(0, ROOT)

METRIC = "256³ projections/s to 1e-6 resid: mixed+graph vs plain FP32; % HBM peak"
UNIT = "projections/s"
WORKLOAD = "whirl256"
TOL = 1e-6
MAXITER = 200
DT = 1.0 / 48
FALLBACK_HBM_GBS = 6650.0


def workload_config(precision, graph):
    return {"workload": "whirl256: 256^3 cylindrical basin (wall r=0.45 N dx, water 0.6 deep, dx=0.05 m), "
                        "Rankine vortex Gamma=225 m^2/s core 2.5 m + uniform[-1,1) m/s faces, seed 1001",
            "cells": 256 ** 3, "tol": TOL, "precision": precision, "graph": graph,
            "l2": "inputs larger than L2 (each CG iteration streams ~1 GB through 126 MB of L2); no flush",
            "parallelism": "replicas"}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel_key):
    """DRAM bytes per launch of the dominant kernel, from the committed ncu summary (or None)."""
    path = os.path.join(ROOT, "profiles", "ncu_whirl256_kernels.md")
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch\[" + re.escape(kernel_key) + r"\]\s*=\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


class ClockSampler:
    """SM clocks and throttle reasons of this process's GPU, sampled through NVML in a
    background thread while the timed region runs (one sample at start, one at stop, and
    every `period_s` between them, so even a 100 ms region has several). The GPU is found
    by its UUID (CUDA and NVML number devices differently under CUDA_VISIBLE_DEVICES)."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, index, period_s=0.01):
        self.index = index
        self.period = period_s
        self.handle = None
        self.err = None
        self.samples = []
        self.thread = None
        self.stop_flag = None
        try:
            import pynvml
            import torch

            self.nvml = pynvml
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(index).uuid)
            uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
            self.handle = pynvml.nvmlDeviceGetHandleByUUID(uuid)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
        except Exception as e:  # no NVML: the line says so
            self.err = f"nvml unavailable: {type(e).__name__}: {e}"

    def _sample(self):
        n = self.nvml
        sm = float(n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM))
        mask = int(n.nvmlDeviceGetCurrentClocksEventReasons(self.handle))
        try:
            watts = n.nvmlDeviceGetPowerUsage(self.handle) / 1000.0
        except Exception:
            watts = None
        self.samples.append((sm, mask, watts))

    def start(self):
        import threading

        if self.handle is None:
            return
        self.samples = []
        self.stop_flag = threading.Event()
        self._sample()

        def loop():
            while not self.stop_flag.wait(self.period):
                try:
                    self._sample()
                except Exception:
                    pass

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def stop(self):
        if self.handle is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.err or "nvml unavailable"], "samples": 0}
        self.stop_flag.set()
        self.thread.join(timeout=5)
        self._sample()
        sm = sorted(x[0] for x in self.samples)
        reasons = set()
        for _, mask, _ in self.samples:
            for name, attr in self.REASONS:
                bit = getattr(self.nvml, attr, 0)
                if bit and mask & bit:
                    reasons.add(name)
        watts = [x[2] for x in self.samples if x[2] is not None]
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": self.max_mhz, "reasons": sorted(reasons),
                "samples": len(sm), "sm_mhz_min": sm[0], "power_w_max": round(max(watts), 1) if watts else None,
                "source": "nvml"}


def dist_init():
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_mpp(args):
    import numpy as np
    import torch

    import mpp
    from mpp import scene

    world, rank, local = dist_init()
    dev = torch.device("cuda", local)
    basin = scene.config_basin(args.workload if args.ncu else WORKLOAD)
    g = basin.grid
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    types, phi = T(basin.types), T(basin.phi)
    u0, v0, w0 = T(basin.u), T(basin.v), T(basin.w)
    u, v, w = u0.clone(), v0.clone(), w0.clone()
    fu, fv, fw = (torch.zeros(a.numel(), dtype=torch.uint8, device=dev) for a in (u0, v0, w0))
    P = torch.zeros(g.ncells, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def make(precision, graph):
        return mpp.Projector(g, tol=TOL, maxiter=MAXITER, precision=precision, graph=graph)

    def timed(proj, steps, warmup, sampler=None):
        vol0 = proj.volume(phi)
        launches, its, last = 0, [], None

        def step():
            nonlocal launches, last
            u.copy_(u0)
            v.copy_(v0)
            w.copy_(w0)
            P.zero_()
            last = proj.project(u, v, w, fu, fv, fw, P, types, phi, vol0, DT)
            return last

        for _ in range(warmup):
            step()
        barrier(world)
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            r = step()
            launches += r.kernel_launches
            its.append(r.iterations)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        clocks = sampler.stop() if sampler else None
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        return ms, launches, its, last, clocks

    prec = args.precision
    if args.ncu:
        # profiling mode: the headline projection only, its CG loop run from the host so a
        # profiler sees each kernel launch (kernels inside the graph's WHILE node are not
        # reported one by one); no timing is printed. --tuned gives the autotuner's choice
        # (fine form, coarse form, sweeps, coarsest sweeps) without running it.
        proj = make(prec, False)
        if args.tuned:
            fine, coarse, sw, swc, csw = args.tuned.split(",")
            forms = {"vector": 0, "tma": 1, "column": 2, "async": 3}
            proj.set(sweeps=int(sw), sweeps_coarse=int(swc), coarse=int(csw))
            proj.lib.mpp_ctx_set_smoothers(proj._ctx, forms[fine], forms[coarse])
        vol0 = proj.volume(phi)
        for _ in range(args.steps):
            u.copy_(u0); v.copy_(v0); w.copy_(w0); P.zero_()
            r = proj.project(u, v, w, fu, fv, fw, P, types, phi, vol0, DT)
        torch.cuda.synchronize()
        print(json.dumps({"ncu_mode": True, "iterations": r.iterations, "status": r.status}), flush=True)
        return

    # headline: mixed precision + graph, smoother forms and sweeps autotuned on this basin
    # (before the timed region)
    proj = make(prec, True)
    tune = proj.autotune(u0, v0, w0, types, phi)
    sampler = ClockSampler(local) if rank == 0 else None
    ms, launches, its, res, clocks = timed(proj, args.steps, args.warmup, sampler)
    P_mixed = P.detach().cpu().numpy().copy()
    value = world * args.steps / (ms / 1e3)
    # the graph's per-iteration time: the same projection with its iterations capped at half,
    # the difference of the two times over the iterations dropped (the rest of a step is the
    # once-per-projection part)
    cap = max(1, its[-1] // 2)
    proj.set(maxiter=cap)
    steps_cap = max(3, args.steps // 2)
    ms_cap, _, its_cap, _, _ = timed(proj, steps_cap, 2)
    proj.set(maxiter=MAXITER)
    graph_it_ms = max(1e-6, (ms / args.steps - ms_cap / steps_cap) / max(1, its[-1] - its_cap[-1]))
    graph_fixed_ms = ms / args.steps - its[-1] * graph_it_ms
    # the in-graph time of one fine-level colour pass of the smoother: projections capped at
    # `cap` iterations with the autotuned fine sweeps and with one fewer (four fine colour
    # passes fewer an iteration, two down and two up), timed back to back; the difference
    # over the passes removed
    sw = int(proj.opts.sweeps)
    fine_pass_ms = None
    if sw > 1:
        proj.set(maxiter=cap)
        ms_a, _, _, _, _ = timed(proj, steps_cap, 2)
        proj.set(maxiter=cap, sweeps=sw - 1)
        ms_b, _, _, _, _ = timed(proj, steps_cap, 2)
        proj.set(maxiter=MAXITER, sweeps=sw)
        fine_pass_ms = max(1e-6, (ms_a - ms_b) / steps_cap / (4 * cap))

    # plain FP32 (the reference's arithmetic and V-cycle settings, host-driven loop)
    proj32 = make("fp32", False)
    ms32, launches32, its32, res32, _ = timed(proj32, args.steps, args.warmup)
    P_fp32 = P.detach().cpu().numpy().copy()
    value32 = world * args.steps / (ms32 / 1e3)
    del proj32
    # FP32 with the graph and its own autotuning: splits the headline's gain into the part
    # precision buys and the part the graph and tuning buy
    proj32g = make("fp32", True)
    tune32 = proj32g.autotune(u0, v0, w0, types, phi)
    ms32g, _, its32g, _, _ = timed(proj32g, args.steps, args.warmup)
    value32g = world * args.steps / (ms32g / 1e3)
    del proj32g

    # FP64 oracle on the GPU: every result's pressure error
    proj64 = make("fp64", True)
    proj64.set(tol=1e-12, maxiter=400)
    _, _, _, res64, _ = timed(proj64, 1, 0)
    P64 = proj64.solution_f64()
    del proj64
    nrm = float(np.linalg.norm(P64))
    err_mixed = float(np.linalg.norm(P_mixed - P64) / nrm)
    err_fp32 = float(np.linalg.norm(P_fp32 - P64) / nrm)

    # e2e: the public API with the basin's arrays in pinned host memory, every step's copies
    # inside the timed region; mpp.pipeline.HostPipeline overlaps step i+1's upload and step
    # i-1's download with step i's solve (three device buffer sets, three streams)
    from mpp.pipeline import HostPipeline, OUT_NAMES

    pin = lambda t: t.detach().cpu().pin_memory()
    h_in = {"u": pin(u0), "v": pin(v0), "w": pin(w0), "types": pin(types), "phi": pin(phi),
            "P": pin(torch.zeros_like(P))}
    shapes = {"u": u0, "v": v0, "w": w0, "fu": fu, "fv": fv, "fw": fw, "P": P}
    h_out = [{k: torch.empty(shapes[k].numel(), dtype=shapes[k].dtype).pin_memory() for k in OUT_NAMES}
             for _ in range(3)]
    pipe = HostPipeline(proj, dev)
    h2d, d2h = HostPipeline.bytes_per_step(h_in, h_out[0])
    vol0 = proj.volume(phi)
    e2e_steps = max(1, min(args.steps, 50))
    ins = [h_in] * e2e_steps
    outs = [h_out[i % 3] for i in range(e2e_steps)]
    pipe.run([h_in] * max(3, min(args.warmup, 6)), [h_out[i % 3] for i in range(max(3, min(args.warmup, 6)))],
             vol0, DT)
    torch.cuda.synchronize()
    barrier(world)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    e2e_res = pipe.run(ins, outs, vol0, DT, stream=stream)
    f1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms_e2e = max_over_ranks(f0.elapsed_time(f1), world)
    e2e_value = world * e2e_steps / (ms_e2e / 1e3)
    # the downloaded result of the last step is the device-resident headline's result
    e2e_ok = all(r.status == 0 for r in e2e_res) and bool(
        np.array_equal(outs[-1]["P"].numpy(), P_mixed))
    del pipe

    # live per-kernel timing (CUDA events on the launching stream), one profiled projection
    proj.profile(True)
    for _ in range(2):
        u.copy_(u0); v.copy_(v0); w.copy_(w0); P.zero_()
        rprof = proj.project(u, v, w, fu, fv, fw, P, types, phi, vol0, DT)
    prof = proj.profile_read()
    proj.profile(False)
    hbm, peak_src = peaks()
    dom = max(prof, key=lambda e: e["ms"])
    per_launch_bytes = dom["bytes"] / dom["launches"]
    isolated_ms = dom["ms"] / dom["launches"]  # one launch bracketed by events (no overlap)
    key = f"{dom['name']}@{dom['level']}"
    # the fine smoother's launch time inside the graph (back-to-back launches with
    # programmatic dependent launch) where it is the dominant kernel, else the bracketed one
    per_launch_ms = fine_pass_ms if (key == "rbgs@0" and fine_pass_ms) else isolated_ms
    achieved = per_launch_bytes / (per_launch_ms / 1e3) / 1e9
    traffic = ncu_traffic(key)
    # bytes per CG iteration (every kernel inside the loop) over the loop's time
    loop_names = ("start", "rbgs", "residual", "restrict", "bottom", "prolong", "dot", "search", "advance")
    loop = [e for e in prof if e["name"] in loop_names]
    nit = max(1, 2 * rprof.iterations)
    it_bytes = sum(e["bytes"] for e in loop) / nit
    it_ms = sum(e["ms"] for e in loop) / nit
    total_prof_ms = sum(e["ms"] for e in prof)

    out = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; no dataset exists)",
        "config": workload_config(prec, True),
        "iterations": its[-1], "true_rel_residual": res.true_rel_residual, "fp64_rel_error": err_mixed,
        "cells_per_s": value * g.ncells,
        "fp32_plain": {"value": round(value32, 3), "unit": UNIT, "ms_per_step": round(ms32 / args.steps, 4),
                       "iterations": its32[-1], "true_rel_residual": res32.true_rel_residual,
                       "fp64_rel_error": err_fp32, "graph": False, "gpu_launches": launches32},
        "mixed_over_fp32": round(value / value32, 3),
        # the split of that gain: the graph and the autotuned sweeps (FP32 + graph + tuned over
        # plain FP32) and the 16-bit storage alone (mixed over FP32 + graph + tuned)
        "gain_split": {"graph_and_tuning": round(value32g / value32, 3), "precision": round(value / value32g, 3)},
        "autotuned": tune["chosen"],
        "autotune_forms_ms": {f"{r['smoother']}/{r['coarse_smoother']}": r["ms"] for r in tune["table"]
                              if (r["sweeps"], r["sweeps_coarse"], r["coarse_sweeps"]) == (2, 0, 40)},
        "fp32_graph_tuned": {"value": round(value32g, 3), "unit": UNIT, "iterations": its32g[-1],
                             "autotuned": tune32["chosen"]},
        "fp64_oracle": {"iterations": res64.iterations, "true_rel_residual": res64.true_rel_residual},
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps, "overlap": "upload i+1 / solve i / download i-1 on three streams",
                "result_matches_device_run": e2e_ok},
        "roofline": {"bound": "hbm", "kernel": key, "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4), "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)"
                     if peak_src == "measured" else "fallback 6.65 TB/s",
                     "traffic": traffic, "algorithmic_bytes_per_launch": per_launch_bytes,
                     "launch_ms": round(per_launch_ms, 5),
                     "launch_ms_source": "in the graph: projections at the autotuned fine sweeps and one fewer, "
                                         "capped at the same iterations, difference over the fine colour passes "
                                         "removed" if per_launch_ms is fine_pass_ms else "one launch bracketed by events",
                     "isolated": {"launch_ms": round(isolated_ms, 5),
                                  "achieved": round(per_launch_bytes / (isolated_ms / 1e3) / 1e9, 1),
                                  "frac": round(per_launch_bytes / (isolated_ms / 1e3) / 1e9 / hbm, 4),
                                  "note": "one launch bracketed by CUDA events in the host-driven loop: no "
                                          "overlap with its neighbours, ramp and drain included"},
                     "share_of_profiled_time": round(dom["ms"] / total_prof_ms, 4)},
        "iteration_roofline": {"bytes_per_iteration": it_bytes,
                               "profiled": {"ms_per_iteration": round(it_ms, 4),
                                            "achieved": round(it_bytes / (it_ms / 1e3) / 1e9, 1),
                                            "frac": round(it_bytes / (it_ms / 1e3) / 1e9 / hbm, 4),
                                            "note": "each kernel timed alone with CUDA events, host loop"},
                               "graph": {"ms_per_iteration": round(graph_it_ms, 4),
                                         "achieved": round(it_bytes / (graph_it_ms / 1e3) / 1e9, 1),
                                         "frac": round(it_bytes / (graph_it_ms / 1e3) / 1e9 / hbm, 4),
                                         "once_per_projection_ms": round(graph_fixed_ms, 4),
                                         "note": "graph projections at the full and at half the iteration "
                                                 "count: the difference over the iterations dropped"},
                               "peak": hbm},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if world > 1 and not args.no_extras:
        # the batched workload partitioned over the ranks (every rank takes part)
        torch.cuda.empty_cache()
        out["batched"] = bench_batched_partitioned(rank, world, max(3, min(args.steps, 10)))
    if rank == 0 and world == 1 and not args.no_extras:
        # the other workloads, each timed on its own (not part of the headline value)
        del proj
        torch.cuda.empty_cache()
        out["batched"] = bench_batched(max(3, min(args.steps, 10)))
        torch.cuda.empty_cache()
        out["adjoint"] = bench_adjoint(max(3, min(args.steps, 10)))
        torch.cuda.empty_cache()
        out["whirlpool384"] = bench_whirlpool(max(3, min(args.steps, 10)))
        torch.cuda.empty_cache()
        out["extrapolate"] = bench_extrapolate(max(3, min(args.steps, 10)))
        torch.cuda.empty_cache()
        out["levelset"] = bench_levelset(max(3, min(args.steps, 10)))
        torch.cuda.empty_cache()
        out["sparse"] = bench_sparse(max(3, min(args.steps, 10)), cpu=not args.no_cpu)
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(basin, max_seconds=args.cpu_seconds)
    if rank == 0:
        if args.profile_out:
            with open(args.profile_out, "w") as f:
                json.dump({"projection_profile": prof, "iterations": rprof.iterations}, f, indent=1)
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def _events():
    import torch

    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def bench_batched(steps):
    """48 basins (edges from {48, 64, 96, 128}), autotuned, one graph launch per batched
    projection: total projections/s, cells/s and per-basin iterations."""
    import torch

    from mpp import scene
    from mpp.batch import Batch

    basins = scene.batch_basins()
    cells = sum(b.grid.ncells for b in basins)
    batch = Batch(basins, tol=TOL, maxiter=MAXITER, precision="fp32")
    tune = batch.autotune()
    init = [{k: a[k].clone() for k in ("u", "v", "w")} for a in batch.arrays]

    def step():
        for a, i0 in zip(batch.arrays, init):
            for k in ("u", "v", "w"):
                a[k].copy_(i0[k])
            a["P"].zero_()
        return batch.project(DT)

    def timed():
        for _ in range(3):
            step()
        torch.cuda.synchronize()
        e0, e1 = _events()
        # the per-step copies of the 48 initial states are timed too (about 1.2 GB moved)
        e0.record()
        for _ in range(steps):
            res = step()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, res

    chosen = batch.max_group
    ms, res = timed()
    groups = batch.groups
    its = [r.iterations for r in res]
    # the other grouping, for comparison: groups of 16 if chains won, else chains
    batch.set_grouped(16 if chosen < 2 else 0)
    ms_other, res_o = timed()
    batch.set_grouped(chosen)
    launches = sum(r.kernel_launches for r in res)
    return {"basins": len(basins), "cells": cells, "projections_per_s": round(len(basins) / (ms / 1e3), 2),
            "cells_per_s": cells / (ms / 1e3), "ms_per_batch": round(ms, 3), "steps": steps,
            "grouping": {"chosen_max_group": chosen, "groups": groups, "autotune_ms": batch.grouping,
                         "other": {"max_group": 16 if chosen < 2 else 0,
                                   "projections_per_s": round(len(basins) / (ms_other / 1e3), 2),
                                   "same_iterations": its == [r.iterations for r in res_o]}},
            "graph_launches_per_batch": 1, "gpu_launches_per_batch": launches,
            "iterations": [r.iterations for r in res], "all_converged": all(r.status == 0 for r in res),
            "max_true_rel_residual": max(r.true_rel_residual for r in res),
            "autotune": {f"{d[0]}x{d[1]}x{d[2]}": v["chosen"] for d, v in tune.items()},
            "edges": [b.grid.n[0] for b in basins], "precision": "fp32"}


def bench_batched_partitioned(rank, world, steps):
    """The batched workload over `world` GPUs (mpp.batch.project_partitioned): each rank
    projects its LPT share of the 48 basins as one batched graph launch per step, autotuned
    on its own GPU; only per-basin results are gathered. Timed on the device between
    barriers, max over ranks."""
    import torch

    from mpp import scene
    from mpp.batch import lpt_partition, basin_cost, project_partitioned, solve_with_batch

    basins = scene.batch_basins()
    ms_box = {}

    def timer(run):
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        ms_box["ms"] = e0.elapsed_time(e1) / steps
        barrier(world)

    solve = lambda b, idx, **kw: solve_with_batch(b, idx, timer=timer, steps=steps, **kw)
    res = project_partitioned(basins, rank, world, solve=solve, dt=DT, tol=TOL, maxiter=MAXITER)
    ms = max_over_ranks(ms_box.get("ms", 0.0), world)
    parts = lpt_partition([basin_cost(b) for b in basins], world)
    cells = sum(b.grid.ncells for b in basins)
    return {"basins": len(basins), "cells": cells, "ranks": world, "projections_per_s": round(len(basins) / (ms / 1e3), 2),
            "cells_per_s": cells / (ms / 1e3), "ms_per_batch": round(ms, 3), "steps": steps,
            "partition": [len(p) for p in parts], "iterations": [r.iterations for r in res],
            "all_converged": all(r.status == 0 for r in res), "timing": "device, max over ranks",
            "precision": "fp32"}


def bench_adjoint(steps):
    """The adjoint at 128^3 (forward project! + its VJP, FP32 and mixed, error against the
    FP64 form's gradient) and the 10-step 96^3 advect + project rollout's reverse pass."""
    import numpy as np
    import torch

    import mpp
    from mpp import scene
    from mpp.rollout import Rollout

    b = scene.box_basin(128, seed=1003)
    rng = np.random.default_rng(1003)
    ustar = [torch.from_numpy(rng.uniform(-1, 1, a.size).astype(np.float32)).cuda() for a in (b.u, b.v, b.w)]
    out = {"workload": "128^3 basin (seed 1003), loss 1/2 |P(u) - u*|^2, u* uniform[-1, 1]"}
    grads = {}
    for prec in ("fp64", "fp32", "fp16"):
        s = mpp.FlipBasin.from_scene(b, tol=1e-11 if prec == "fp64" else TOL, maxiter=300, precision=prec,
                                     graph=True)
        u0 = [a.clone() for a in (s.u, s.v, s.w)]
        mu = torch.zeros(b.grid.ncells, dtype=torch.float32, device="cuda")

        def fwd():
            for a, x in zip((s.u, s.v, s.w), u0):
                a.copy_(x)
            s.P.zero_()
            return s.projector.project(s.u, s.v, s.w, s.fu, s.fv, s.fw, s.P, s.types, s.phi, s.volume0, DT)

        cot = [torch.empty_like(a) for a in u0]

        def bwd():
            for c, a, t in zip(cot, (s.u, s.v, s.w), ustar):
                torch.sub(a, t, out=c)
            mu.zero_()
            return s.projector.project_vjp(*cot, mu, s.types, s.phi)

        for _ in range(2):
            fwd()
            rb = bwd()
        torch.cuda.synchronize()
        n = 1 if prec == "fp64" else steps
        e0, e1, e2 = _events() + (torch.cuda.Event(enable_timing=True),)
        tf = tb = 0.0
        for _ in range(n):
            e0.record()
            fwd()
            e1.record()
            rb = bwd()
            e2.record()
            torch.cuda.synchronize()
            tf += e0.elapsed_time(e1)
            tb += e1.elapsed_time(e2)
        grads[prec] = np.concatenate([c.cpu().numpy().astype(np.float64) for c in cot])
        if prec != "fp64":
            ref = grads["fp64"]
            out[prec] = {"forward_ms": round(tf / n, 3), "vjp_ms": round(tb / n, 3),
                         "vjp_iterations": rb.iterations,
                         "rel_error_vs_fp64_gradient": float(np.linalg.norm(grads[prec] - ref) / np.linalg.norm(ref))}
        del s
        torch.cuda.empty_cache()
    # rollout
    b96 = scene.box_basin(96, seed=1005)
    u96 = [torch.from_numpy(scene.uniform(1005, 20 + a, int(np.prod(b96.grid.face_shape(a))))).cuda()
           for a in range(3)]
    star = [torch.from_numpy(rng.uniform(-1, 1, a.numel()).astype(np.float32)).cuda() for a in u96]
    s = mpp.FlipBasin.from_scene(b96, tol=TOL, maxiter=MAXITER, precision="fp32", graph=True)
    ro = Rollout(s, 10, 0.02)
    for _ in range(2):
        fin = ro.forward(*u96)
        ro.backward(*[a - t for a, t in zip(fin, star)])
    torch.cuda.synchronize()
    e0, e1, e2 = _events() + (torch.cuda.Event(enable_timing=True),)
    e0.record()
    fin = ro.forward(*u96)
    e1.record()
    g = ro.backward(*[a - t for a, t in zip(fin, star)])
    e2.record()
    torch.cuda.synchronize()
    out["rollout_96_10_steps"] = {"forward_ms": round(e0.elapsed_time(e1), 3), "backward_ms": round(e1.elapsed_time(e2), 3),
                                  "iterations": ro.iterations, "adjoint_iterations": ro.adjoint_iterations,
                                  "checkpoints_bytes": sum(c.numel() * 4 for ck in ro.ckpt for c in ck),
                                  "grad_finite": bool(all(torch.isfinite(a).all() for a in g))}
    return out


def bench_extrapolate(steps):
    """extrapolate!(s; layers = 6) after the 256^3 whirlpool's projection, as step! runs it
    (src/flip.jl:1403-1404): ms a call, and HBM GB/s at the bytes the reach-code design must
    move: a flag read and a code written a face in the first pass, a code read a face a
    layer, a code read and a flag written a face in the last pass, and 4 bytes for each value
    written (the faces a layer reaches and the faces zeroed); neighbours come through the
    caches. `reference_pass_gbs` is the same
    time at the reference's ping-pong structure (10 bytes a face a layer). The projected
    arrays are restored before each call, outside the timed events; the three arrays' faces
    and flags (253 MB) are larger than L2."""
    import torch

    import mpp
    from mpp import scene

    b = scene.config_basin("whirl256")
    s = mpp.FlipBasin.from_scene(b, tol=TOL, maxiter=MAXITER, precision="fp16", graph=True)
    mpp.project(s, DT)
    arrs = (s.u, s.v, s.w, s.fu, s.fv, s.fw)
    saved = [a.clone() for a in arrs]
    layers = 6

    def call():
        for a, x in zip(arrs, saved):
            a.copy_(x)
        e0, e1 = _events()
        e0.record()
        s.projector.extrapolate(*arrs, layers=layers)
        e1.record()
        return e0, e1

    for _ in range(3):
        call()
    ev = [call() for _ in range(steps)]
    torch.cuda.synchronize()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev) / steps
    faces = sum(int(a.numel()) for a in (s.u, s.v, s.w))
    reached = sum(int(torch.count_nonzero(f)) for f in (s.fu, s.fv, s.fw))
    flagged = sum(int(torch.count_nonzero(f)) for f in saved[3:])
    hbm, src = peaks()
    nbytes = faces * (layers + 4) + 4 * ((reached - flagged) + (faces - reached))
    gbs = nbytes / (ms / 1e3) / 1e9
    return {"workload": "whirl256 after its projection (fp16 graph), layers 6", "faces": faces,
            "flagged_before": flagged, "reached_after": reached, "ms": round(ms, 4), "launches": layers + 2,
            "algorithmic_bytes": nbytes, "achieved_gbs": round(gbs, 1), "peak_gbs": hbm,
            "frac": round(gbs / hbm, 4), "peak_source": src,
            "reference_pass_gbs": round(10.0 * faces * layers / (ms / 1e3) / 1e9, 1), "steps": steps}


def bench_levelset(steps):
    """step!'s level-set phase before the projection (src/flip.jl:1399-1401) on the 256^3
    whirlpool: redistance! (band + 3 = 7 Jacobi sweeps, classify! fused into the last) and
    filltrapped! (device-side round loop), each timed with CUDA events. The level set is the
    basin's, made wavy and noisy with sealed air pockets under the surface, so the sweeps
    have surface, far-field and clamped cells and the fill has pockets to fill. Algorithmic
    bytes: a sweep reads and writes phi once (8 bytes a cell), classify! writes a class
    (1); filltrapped! reads the classes once (1), keeps a bit a cell for the air and the
    reached cells (0.25 written, 0.25 read by the fill) and rewrites the cells it fills."""
    import numpy as np
    import torch

    import mpp
    from mpp import scene

    b = scene.config_basin("whirl256")
    g = b.grid
    n1, n2, n3 = g.n
    rng = np.random.default_rng(1001)
    phi = b.phi.reshape(n3, n2, n1) + (0.3 * np.sin(0.2 * np.arange(n1))[None, None, :] * g.dx)
    phi = (phi + rng.uniform(-0.2, 0.2, phi.shape) * g.dx).astype(np.float32)
    types = b.types.reshape(n3, n2, n1).copy()
    types[(types == scene.LIQUID) & (rng.random(types.shape) < 0.02)] = scene.AIR
    phi[types == scene.AIR] = np.abs(phi[types == scene.AIR])
    dev = torch.device("cuda")
    phi0_h = torch.from_numpy(phi.reshape(-1)).to(dev)
    types0_h = torch.from_numpy(types.reshape(-1)).to(dev)
    p = mpp.Projector(g)
    d_phi, d_phi0 = phi0_h.clone(), torch.empty_like(phi0_h)
    d_types = types0_h.clone()
    it = 7
    N = g.ncells

    def run():
        d_phi.copy_(phi0_h)
        d_types.copy_(types0_h)
        e0, e1, e2 = _events() + (torch.cuda.Event(enable_timing=True),)
        e0.record()
        out = p.redistance(d_phi, d_phi0, it, types=d_types)
        e1.record()
        p.filltrapped(d_types, out, 32, rounds=False)
        e2.record()
        return e0, e1, e2

    for _ in range(3):
        run()
    ev = [run() for _ in range(steps)]
    torch.cuda.synchronize()
    ms_r = sum(a.elapsed_time(b_) for a, b_, _ in ev) / steps
    ms_f = sum(b_.elapsed_time(c) for _, b_, c in ev) / steps
    d_phi.copy_(phi0_h)
    out = p.redistance(d_phi, d_phi0, it, types=d_types)
    classified = d_types.clone()
    rounds = p.filltrapped(d_types, out, 32)
    filled = int(torch.count_nonzero(d_types != classified))
    hbm, src = peaks()
    bytes_r = N * (8.0 * it + 1.0)
    bytes_f = N * (1.0 + 0.5) + 5.0 * filled
    return {"workload": "whirl256 level set (wavy, noisy, 2% of the water made air pockets)", "cells": N,
            "redistance_sweeps": it, "redistance_classify_ms": round(ms_r, 4),
            "redistance_gbs": round(bytes_r / (ms_r / 1e3) / 1e9, 1),
            "redistance_frac": round(bytes_r / (ms_r / 1e3) / 1e9 / hbm, 4),
            "filltrapped_ms": round(ms_f, 4), "filltrapped_rounds": rounds, "cells_filled": filled,
            "filltrapped_gbs": round(bytes_f / (ms_f / 1e3) / 1e9, 1), "peak_gbs": hbm, "peak_source": src,
            "steps": steps}


def bench_sparse(steps, cpu=True):
    """The sparse two-resolution basin's project! (src/sflip.jl:1998-2018): the seeded
    whirlpool of mpp.sparse_scene.charybdis, 32 x 32 x 16 blocks of 16^3 cells (a 512 x 512 x
    256 fine-cell box over a 128 x 128 x 64 coarse grid), 2948 fine blocks along the funnel
    (12.1 M fine cells, 5.1 M of them water), in the reference's Float32 arithmetic with
    pressure!'s defaults (tol 1e-4, one sweep pair, boost 1), the CG loop driven from the host.
    Each call restores P and the velocities outside its CUDA events. Beside it: the level-0
    stencil pass (apply!: the composite operator over every fine block and the coarse grid,
    one launch) timed alone, its achieved GB/s on the bytes it must move (a fine cell of the
    slots in use: x 4, packed couplings 2, diagonal 4, q 4; a coarse cell: activity 1 and q 4,
    and for an active one x 4, b-side diagonal 4 and six couplings 24), and the CPU oracle's
    projection of the same basin on the host's threads."""
    import numpy as np
    import torch

    from mpp import sparse as msp
    from mpp import sparse_scene as ss

    sc = ss.charybdis()
    # the CG loop driven from the host, one state read an iteration: faster here than the
    # graph's conditional loop (10.8 against 11.3 ms measured)
    s = msp.SparseBasin.from_scene(sc, graph=False, tol=1e-4, maxiter=200)
    saved = {k: getattr(s, k).clone() for k in ("Pf", "Pc", "uf", "uc", "vf", "vc", "wf", "wc")}

    def call():
        for k, v in saved.items():
            getattr(s, k).copy_(v)
        e0, e1 = _events()
        e0.record()
        msp.project(s, DT)
        e1.record()
        return e0, e1

    for _ in range(3):
        call()
    ev = [call() for _ in range(steps)]
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev) / steps
    its = s.iterations[-1]
    # the level-0 stencil pass alone
    used = int((sc.where[:, 0] >= 0).sum())
    fine_u = (sc.tf == 1) & np.repeat(sc.where[:, 0] >= 0, 4096)
    ncc = int(np.prod(sc.grid.nc))
    rng = np.random.default_rng(5)
    xf = torch.from_numpy(np.where(fine_u, rng.standard_normal(fine_u.size), 0).astype(np.float32)).cuda()
    xc = torch.from_numpy(np.where(sc.tc == 1, rng.standard_normal(ncc), 0).astype(np.float32)).cuda()
    qf, qc = torch.empty_like(xf), torch.empty_like(xc)
    s.operator()
    cact = int(s.read("act_c").astype(bool).sum())
    for _ in range(3):
        s.apply(xf, xc, qf, qc)
    n_apply = 20
    e0, e1 = _events()
    e0.record()
    for _ in range(n_apply):
        s.apply(xf, xc, qf, qc)
    e1.record()
    torch.cuda.synchronize()
    apply_ms = e0.elapsed_time(e1) / n_apply
    nbytes = used * 4096 * 14 + ncc * 5 + cact * 32
    hbm, src = peaks()
    out = {"workload": "sparse whirlpool (charybdis): 32x32x16 blocks, 2948 fine blocks, coarse 128x128x64, tol 1e-4",
           "fine_blocks": used, "fine_cells": used * 4096, "fine_water_cells": int(fine_u.sum()),
           "coarse_cells": ncc, "ms_per_projection": round(ms, 3), "projections_per_s": round(1e3 / ms, 2),
           "iterations": its, "rel_residual": s.last.rel_residual, "graph": False,
           "kernel_launches": int(s.last.kernel_launches),
           "apply_pass": {"ms": round(apply_ms, 4), "algorithmic_bytes": nbytes,
                          "achieved_gbs": round(nbytes / (apply_ms / 1e3) / 1e9, 1), "peak_gbs": hbm,
                          "frac": round(nbytes / (apply_ms / 1e3) / 1e9 / hbm, 4), "peak_source": src},
           "steps": steps}
    del s
    torch.cuda.empty_cache()
    if cpu:
        import oracle
        from oracle import sparse as osp

        vol = osp.volume(sc)
        t0 = time.perf_counter()
        info = osp.project(sc.copy(), vol, tol=1e-4, maxiter=200)
        cpu_s = time.perf_counter() - t0
        out["cpu_oracle"] = {"ms_per_projection": round(cpu_s * 1e3, 1), "iterations": info["iterations"],
                             "threads": oracle.num_threads(), "kind": "port",
                             "sample": "one projection of the same basin by the C/OpenMP oracle"}
    return out


def run_sparse_ncu(steps):
    """The sparse workload's projections with the CG loop driven from the host (every kernel
    its own launch, for a profiler's launch list); each starts from the same P and velocities."""
    import torch

    from mpp import sparse as msp
    from mpp import sparse_scene as ss

    sc = ss.charybdis()
    s = msp.SparseBasin.from_scene(sc, graph=False, tol=1e-4, maxiter=200)
    saved = {k: getattr(s, k).clone() for k in ("Pf", "Pc", "uf", "uc", "vf", "vc", "wf", "wc")}
    for _ in range(max(1, steps)):
        for k, v in saved.items():
            getattr(s, k).copy_(v)
        msp.project(s, DT)
    torch.cuda.synchronize()
    print(json.dumps({"sparse_ncu": True, "iterations": s.iterations, "launches": int(s.last.kernel_launches)}))


def bench_whirlpool(steps):
    """384 x 384 x 256 whirlpool, mixed precision with the FGMRES fallback to 1e-6: projections/s,
    the FP64 form's pressure error, and achieved HBM GB/s per kernel family."""
    import numpy as np
    import torch

    import mpp
    from mpp import scene

    b = scene.config_basin("whirlpool384")
    s64 = mpp.FlipBasin.from_scene(b, tol=1e-11, maxiter=400, precision="fp64", graph=True)
    mpp.project(s64, DT)
    P64 = s64.projector.solution_f64()
    del s64
    torch.cuda.empty_cache()
    s = mpp.FlipBasin.from_scene(b, tol=TOL, maxiter=MAXITER, precision="fp16", graph=True, fallback=True)
    u0 = [a.clone() for a in (s.u, s.v, s.w)]

    def step():
        for a, x in zip((s.u, s.v, s.w), u0):
            a.copy_(x)
        s.P.zero_()
        return s.projector.project(s.u, s.v, s.w, s.fu, s.fv, s.fw, s.P, s.types, s.phi, s.volume0, DT)

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for _ in range(steps):
        r = step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    err = float(np.linalg.norm(s.P.cpu().numpy() - P64) / np.linalg.norm(P64))
    s.projector.profile(True)
    step()
    prof = s.projector.profile_read()
    s.projector.profile(False)
    fam = {}
    for e in prof:
        f = fam.setdefault(e["name"], [0.0, 0.0])
        f[0] += e["bytes"]
        f[1] += e["ms"]
    per_kernel = {k: round(v[0] / (v[1] / 1e3) / 1e9, 1) for k, v in sorted(fam.items(), key=lambda kv: -kv[1][1])
                  if v[1] > 0}
    return {"cells": b.grid.ncells, "projections_per_s": round(1e3 / ms, 3), "ms_per_projection": round(ms, 3),
            "iterations": r.iterations, "fallback_used": r.fallback_used, "status": r.status,
            "true_rel_residual": r.true_rel_residual, "fp64_rel_error": err, "precision": "fp16",
            "achieved_gbs_by_kernel": per_kernel, "steps": steps}


def cpu_baseline(basin, max_seconds=30.0):
    """The oracle (the reference's FP32 projection restated in C + OpenMP) on this host."""
    import oracle

    threads = oracle.num_threads()
    vol0 = oracle.volume(basin.grid, basin.phi)
    t0 = time.perf_counter()
    n = 0
    while True:
        oracle.project(basin, volume0=vol0, dt=DT, tol=TOL, maxiter=MAXITER)
        n += 1
        el = time.perf_counter() - t0
        if el * (n + 1) / n > max_seconds:
            break
    return {"value": round(n / el, 4), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} full whirl256 projection(s) (256^3, tol 1e-6) by the C/OpenMP oracle, {el:.1f} s"}


def run_reference(args):
    """The reference arm: the oracle's projection on the host cores (rank 0 only)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    import oracle
    from mpp import scene

    basin = scene.config_basin(WORKLOAD)
    threads = oracle.num_threads()
    vol0 = oracle.volume(basin.grid, basin.phi)
    run = lambda: oracle.project(basin, volume0=vol0, dt=DT, tol=TOL, maxiter=MAXITER)
    warm = max(1, args.warmup)  # W warm-up projections, untimed (each takes seconds on the CPU)
    t0 = time.perf_counter()
    for _ in range(warm):
        run()
    first = (time.perf_counter() - t0) / warm
    budget = args.reference_seconds
    steps = max(1, min(args.steps, int(budget / max(first, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(steps):
        info = run()["info"]
    el = time.perf_counter() - t0
    value = steps / el
    out = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "steps_timed": steps, "warmup": warm, "ms_per_step": round(1e3 * el / steps, 2), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; no dataset exists)",
           "impl": "reference", "config": workload_config("fp32", False), "iterations": info.iterations,
           "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": f"{steps} full whirl256 projection(s) timed (of {args.steps} asked, within "
                                      f"{budget:.0f} s) after {warm} warm-up(s), C/OpenMP restatement of src/flip.jl"
                                      f":1144-1156 (the Julia/Vulkan reference cannot run here)"},
           "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="mpp", choices=["mpp", "reference"])
    ap.add_argument("--precision", default="fp16", choices=["fp16", "bf16", "fp32"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched, adjoint and whirlpool workloads")
    ap.add_argument("--cpu-seconds", type=float, default=25.0)
    ap.add_argument("--reference-seconds", type=float, default=150.0)
    ap.add_argument("--profile-out", default=None)
    ap.add_argument("--tuned", default=None,
                    help="--ncu mode: fine,coarse,sweeps,coarse-level sweeps,coarsest (e.g. vector,column,4,2,10)")
    ap.add_argument("--ncu", action="store_true",
                    help="profiling mode: --steps headline projections from the host loop, nothing timed")
    ap.add_argument("--workload", default=WORKLOAD, choices=[WORKLOAD, "plain64", "box128"],
                    help="--ncu mode: the basin profiled (a smaller one to size a capture)")
    ap.add_argument("--sparse-ncu", action="store_true",
                    help="profiling mode: --steps projections of the sparse workload from the host loop, nothing timed")
    args = ap.parse_args()
    if args.sparse_ncu:
        run_sparse_ncu(args.steps)
        return
    if args.warmup < 3 and args.impl == "mpp" and not args.ncu:
        ap.error("--warmup must be at least 3")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_mpp(args)


if __name__ == "__main__":
    main()
