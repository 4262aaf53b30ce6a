"""The V-cycle's small levels run in one thread-block cluster (k_cmg: levels of 32^3 cells
and fewer, resident in the cluster's shared memory) or as per-level launches
(MPP_CMG=0). With the same one-CTA bottom bound (MPP_BOTTOM_CELLS=512 for both), every
pass computes the same arithmetic in the same order, so a projection must agree bit for
bit, iteration count included, in every precision form."""
import os

import numpy as np
import pytest

from mpp import scene

pytestmark = pytest.mark.gpu


def _solve(basin, precision, cluster):
    import mpp

    saved = {k: os.environ.get(k) for k in ("MPP_CMG", "MPP_BOTTOM_CELLS")}
    os.environ["MPP_BOTTOM_CELLS"] = "512"
    if cluster:
        os.environ.pop("MPP_CMG", None)
    else:
        os.environ["MPP_CMG"] = "0"
    try:  # the context reads both when it is created
        s = mpp.FlipBasin.from_scene(basin, tol=1e-6, maxiter=100, precision=precision, graph=True)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    if cluster:
        s.projector.profile(True)  # to see the cluster kernel launch (the loop then runs from the host)
    mpp.project(s, 1 / 48)
    launched = {e["name"] for e in s.projector.profile_read()} if cluster else set()
    return s.P.cpu().numpy(), s.u.cpu().numpy(), s.last.iterations, launched


@pytest.mark.parametrize("name", ["box64", "whirl256"])
@pytest.mark.parametrize("precision", ["fp16", "bf16", "fp32"])
def test_cluster_matches_per_level(cuda, name, precision):
    b = scene.config_basin(name)
    P0, u0, it0, _ = _solve(b, precision, cluster=False)
    P1, u1, it1, launched = _solve(b, precision, cluster=True)
    assert "cluster" in launched, launched
    assert it1 == it0
    assert np.array_equal(P1.view(np.uint32), P0.view(np.uint32))
    assert np.array_equal(u1.view(np.uint32), u0.view(np.uint32))
