"""HostPipeline: projections of host-resident states, copies overlapped with the solves.

Each state's result, downloaded by the pipeline, must equal the same projection run on
device-resident arrays (the same kernels on the same inputs: bit for bit), whatever the
number of states in flight relative to the pipeline's three buffer sets.
"""
import numpy as np
import pytest

from mpp import scene

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("count", [1, 2, 5])
def test_pipeline_matches_device_projection(cuda, count):
    import torch

    import mpp
    from mpp.pipeline import OUT_NAMES, HostPipeline

    base = scene.box_basin(32, seed=4321)
    g = base.grid
    states = []
    for i in range(count):
        b = base.copy()
        for a, arr in enumerate((b.u, b.v, b.w)):
            arr[:] = scene.uniform(900 + i, a, arr.size)
            scene.solidify(g, arr, a)
        states.append(b)
    proj = mpp.Projector(g, tol=1e-6, maxiter=100, graph=True)
    vol0 = proj.volume(torch.from_numpy(base.phi).to(cuda)) * 1.001
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    ins = [{"u": pin(b.u), "v": pin(b.v), "w": pin(b.w), "types": pin(b.types), "phi": pin(b.phi),
            "P": pin(np.zeros(g.ncells, np.float32))} for b in states]
    shapes = {"u": b.u, "v": b.v, "w": b.w, "P": np.zeros(g.ncells, np.float32)}
    outs = []
    for _ in states:
        o = {k: torch.empty(shapes[k].size, dtype=torch.float32).pin_memory() for k in ("u", "v", "w", "P")}
        o.update({f: torch.empty(shapes[f[1]].size, dtype=torch.uint8).pin_memory() for f in ("fu", "fv", "fw")})
        outs.append(o)
    pipe = HostPipeline(proj, cuda)
    res = pipe.run(ins, outs, vol0, 1 / 48)
    torch.cuda.synchronize()
    assert len(res) == count
    for i, b in enumerate(states):
        s = mpp.FlipBasin.from_scene(b, tol=1e-6, maxiter=100, graph=True)
        s.volume0 = vol0
        mpp.project(s, 1 / 48)
        assert res[i].status == 0 and res[i].iterations == s.iterations[-1]
        for k in OUT_NAMES:
            np.testing.assert_array_equal(outs[i][k].numpy(), getattr(s, k).cpu().numpy(), err_msg=f"state {i} {k}")


def test_pipeline_rejects_pageable_host_memory(cuda):
    import torch

    import mpp
    from mpp.pipeline import HostPipeline

    b = scene.box_basin(16, seed=5)
    proj = mpp.Projector(b.grid)
    pipe = HostPipeline(proj, cuda)
    ins = [{"u": torch.from_numpy(b.u)}]
    with pytest.raises(ValueError, match="page-locked"):
        pipe.run(ins, [{}], 1.0, 1 / 48)
