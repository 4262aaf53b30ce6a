"""Build libmpp.so in-tree: nvcc for sm_100a only, no JIT, no torch extension machinery.

    python maelstrom.jl_b200/build.py [--verbose]

``-fmad=false`` keeps every a*b+c as two roundings, so the FP32 kernels round exactly
as the reference's Float32 code; the kernels are bandwidth-bound, so the lost FMA
throughput costs nothing measurable.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libmpp.so")
SOURCES = ["mpp.cu", "mpp_sparse.cu"]
HEADERS = ["mpp_common.cuh", "mpp_base.cuh", "mpp_tiles.cuh", "mpp_stream.cuh", "mpp_tma.cuh", "mpp_fgmres.cuh", "mpp_adjoint.cuh", "mpp_advect.cuh", "mpp_cmg.cuh", "mpp_extrap.cuh", "mpp_levelset.cuh", "mpp_group.cuh", "mpp_sparse.cuh"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def flags(verbose: bool = False) -> list:
    f = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
         "-Xcompiler", "-fPIC,-O2", "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    if verbose:
        f += ["-Xptxas", "-v"]
    return f


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "mpp.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and not stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    # each translation unit compiles in its own nvcc process, in parallel; then one link
    objs, procs = [], []
    for src in SOURCES:
        obj = os.path.join(LIBDIR, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc()] + flags(verbose) + ["-c", "-o", obj, os.path.join(CSRC, src)]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        objs.append(obj)
    for cmd, p in procs:
        out, err = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed ({p.returncode}):\n{' '.join(cmd)}\n{out}\n{err}")
        if verbose:
            sys.stderr.write(out + err)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp] + objs
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({res.returncode}):\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    for o in objs:
        os.remove(o)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
