"""The large whirlpool: 384 x 384 x 256 cells, Rankine vortex, free surface lowered by its
cyclostrophic profile (a dry throat), eddy noise in the outer tenth of the radius. Mixed
precision with the FGMRES fallback to 1e-6, against the FP64 form on the GPU."""
import numpy as np
import pytest

from mpp import scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def whirlpool():
    return scene.config_basin("whirlpool384")


def test_whirlpool_geometry(whirlpool):
    b = whirlpool
    assert b.grid.n == (384, 384, 256) and b.grid.levels == 7
    # the throat reaches the floor: no liquid on the axis at the bottom
    n1, n2, _ = b.grid.n
    t = b.types.reshape(256, n2, n1)
    assert t[0, n2 // 2, n1 // 2] != scene.LIQUID
    assert 0.1 < b.liquid_fraction < 0.6


@pytest.mark.parametrize("precision", ["fp16", "bf16", "fp32"])
def test_whirlpool_converges(cuda, whirlpool, precision):
    import torch

    import mpp

    b = whirlpool
    s64 = mpp.FlipBasin.from_scene(b, tol=1e-11, maxiter=400, precision="fp64", graph=True)
    mpp.project(s64, 1 / 48)
    P64 = s64.projector.solution_f64()
    del s64
    torch.cuda.empty_cache()
    s = mpp.FlipBasin.from_scene(b, tol=1e-6, maxiter=100, precision=precision, graph=True, fallback=True)
    mpp.project(s, 1 / 48)
    r = s.last
    assert r.status == 0 and r.true_rel_residual <= 1e-6, r.as_dict()
    P = s.P.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(P - P64) / np.linalg.norm(P64) <= 1e-4
