"""mpp_extrapolate (extrapolate!, src/flip.jl:1192-1206) against the oracle, bit for bit:
on random flags and velocities at every layer count the reference's callers use (and 0,
1, 2 for the ping-pong edge cases), and on the projection's own output at 64^3 and at the
256^3 whirlpool with step!'s 6 layers (:1404)."""
import numpy as np
import pytest

import oracle
from mpp import scene

pytestmark = pytest.mark.gpu


def _dev(a, dtype):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _run(proj, vel, fl, layers):
    import torch

    tv = [_dev(a, np.float32) for a in vel]
    tf = [_dev(a, np.uint8) for a in fl]
    proj.extrapolate(*tv, *tf, layers=layers)
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in tv] + [t.cpu().numpy() for t in tf]


def _same(got, want):
    for x, y in zip(got, want):
        assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))


@pytest.mark.parametrize("layers", [0, 1, 2, 3, 4, 6])
@pytest.mark.parametrize("density", [0.02, 0.3])
def test_random_flags_match_oracle(cuda, layers, density):
    import mpp

    b = scene.box_basin((48, 48, 32), seed=5100)
    g = b.grid
    rng = np.random.default_rng(7 + layers)
    vel = [rng.uniform(-1, 1, int(np.prod(g.face_shape(a)))).astype(np.float32) for a in range(3)]
    fl = [(rng.random(int(np.prod(g.face_shape(a)))) < density).astype(np.uint8) for a in range(3)]
    s = mpp.FlipBasin.from_scene(b)
    _same(_run(s.projector, vel, fl, layers), oracle.extrapolate(g, *vel, *fl, layers=layers))


@pytest.mark.parametrize("name,precision", [("box64", "fp32"), ("whirl256", "fp16")])
def test_after_projection_matches_oracle(cuda, name, precision):
    import mpp

    b = scene.config_basin(name)
    s = mpp.FlipBasin.from_scene(b, tol=1e-6, maxiter=100, precision=precision, graph=True)
    mpp.project(s, 1 / 48)
    vel = [t.cpu().numpy() for t in (s.u, s.v, s.w)]
    fl = [t.cpu().numpy() for t in (s.fu, s.fv, s.fw)]
    want = oracle.extrapolate(b.grid, *vel, *fl, layers=6)
    mpp.extrapolate(s, layers=6)
    got = [t.cpu().numpy() for t in (s.u, s.v, s.w, s.fu, s.fv, s.fw)]
    _same(got, want)
    assert sum(int(np.count_nonzero(f)) for f in got[3:]) > sum(int(np.count_nonzero(f)) for f in fl)


def test_overlapping_arrays_are_refused(cuda):
    import mpp

    b = scene.box_basin(16, seed=5101)
    s = mpp.FlipBasin.from_scene(b)
    with pytest.raises(Exception, match="overlap"):
        s.projector.extrapolate(s.u, s.u, s.w, s.fu, s.fv, s.fw, layers=2)


def test_too_many_layers_are_refused(cuda):
    import mpp

    b = scene.box_basin(16, seed=5102)
    s = mpp.FlipBasin.from_scene(b)
    with pytest.raises(Exception, match="layers"):
        s.projector.extrapolate(s.u, s.v, s.w, s.fu, s.fv, s.fw, layers=255)
