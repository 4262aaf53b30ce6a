"""Advection (mpp_advect, mpp_advect_phi), its adjoint (mpp_advect_vjp) and rollouts of
advect + project on the GPU, against the oracle."""
import numpy as np
import pytest

import oracle
from mpp import scene

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _np(t):
    return t.detach().cpu().numpy()


def _flow(g, seed, scale=1.0):
    return [(scene.uniform(seed, 20 + a, int(np.prod(g.face_shape(a)))) * scale).astype(np.float32) for a in range(3)]


@pytest.mark.parametrize("n,scale", [(16, 1.0), (32, 4.0), (64, 0.5), (64, 12.0)])
def test_advect_bitexact(cuda, n, scale):
    import mpp

    b = scene.box_basin(n, seed=5000 + n)
    g = b.grid
    us = _flow(g, 50 + n, scale)
    p = mpp.Projector(g)
    outs = p.advect(*(_t(a, cuda) for a in us), 0.02)
    for got, want in zip(outs, oracle.advect_velocity(g, *us, 0.02)):
        np.testing.assert_array_equal(_np(got), want)
    phi = _np(p.advect_phi(_t(b.phi, cuda), *(_t(a, cuda) for a in us), 0.02))
    np.testing.assert_array_equal(phi, oracle.advect(g, b.phi, None, *us, 0.02))


@pytest.mark.parametrize("n,scale", [(16, 1.0), (32, 4.0)])
def test_advect_vjp_matches_oracle(cuda, n, scale):
    import mpp

    b = scene.box_basin(n, seed=5100 + n)
    g = b.grid
    us = _flow(g, 60 + n, scale)
    rng = np.random.default_rng(n)
    gs = [rng.uniform(-1, 1, a.size).astype(np.float32) for a in us]
    p = mpp.Projector(g)
    got = np.concatenate([_np(a) for a in p.advect_vjp(*(_t(a, cuda) for a in gs), *(_t(a, cuda) for a in us), 0.02)])
    want32 = np.concatenate(oracle.advect_velocity_vjp(g, *gs, *us, 0.02))
    want64 = np.concatenate(oracle.advect_velocity_vjp(g, *gs, *us, 0.02, prec=64))
    # same Float32 trajectories as the FP32 oracle; only the order of the sums differs
    assert np.abs(got - want32).max() <= 1e-5 * np.abs(want32).max()
    # against FP64 trajectories: a node whose Float32 path lands on the other side of a
    # cell face or clamp than the FP64 one differs locally (a kink of trilinear)
    assert np.linalg.norm(got - want64) / np.linalg.norm(want64) <= 1e-3


def _rollout_case(n, steps, seed):
    b = scene.box_basin(n, seed=seed)
    us = _flow(b.grid, seed + 1)
    rng = np.random.default_rng(seed)
    ustar = [rng.uniform(-1, 1, a.size).astype(np.float32) for a in us]
    return b, us, ustar


@pytest.mark.parametrize("steps,bound", [(3, 1e-4), (10, 1e-3)])
def test_rollout_gradient_matches_fp64_oracle(cuda, steps, bound):
    """32^3 rollout, FP32 on the GPU against the FP64 oracle's reverse pass. Trajectories
    that cross a cell face on one side of the rounding and not the other add local kinks,
    more of them the longer the rollout."""
    import mpp
    from mpp.rollout import Rollout

    b, us, ustar = _rollout_case(32, steps, 5200 + steps)
    s = mpp.FlipBasin.from_scene(b, tol=1e-6, maxiter=200, graph=True)
    ro = Rollout(s, steps, 0.02)
    fin = ro.forward(*(_t(a, cuda) for a in us))
    cot = [a - _t(t, cuda) for a, t in zip(fin, ustar)]
    grad = np.concatenate([_np(a).astype(np.float64) for a in ro.backward(*cot)])
    vol0 = oracle.volume(b.grid, b.phi)
    st = oracle.rollout(b, *us, steps, 0.02, volume0=vol0)
    for a, c in zip(st[-1], ro.ckpt[-1]):
        assert np.abs(_np(c) - a).max() <= 1e-4 * np.abs(a).max()
    cot64 = [a - t.astype(np.float64) for a, t in zip(st[-1], ustar)]
    want = np.concatenate(oracle.rollout_vjp(b, st, *cot64, 0.02))
    assert np.linalg.norm(grad - want) / np.linalg.norm(want) <= bound
    assert len(ro.iterations) == steps and len(ro.adjoint_iterations) == steps


def test_autograd_rollout_equals_explicit(cuda):
    """advect + project under torch.autograd gives the explicit reverse pass."""
    import torch

    import mpp
    from mpp import adjoint, rollout

    b, us, ustar = _rollout_case(32, 3, 5300)
    s1 = mpp.FlipBasin.from_scene(b, tol=1e-6, maxiter=200)
    x = [_t(a, cuda).requires_grad_(True) for a in us]
    y = x
    for _ in range(3):
        y = rollout.advect(*y, s1, 0.02)
        y = adjoint.project(*y, s1, 0.02)
    loss = 0.5 * sum(((a - _t(t, cuda)) ** 2).sum() for a, t in zip(y, ustar))
    loss.backward()
    s2 = mpp.FlipBasin.from_scene(b, tol=1e-6, maxiter=200)
    ro = rollout.Rollout(s2, 3, 0.02)
    fin = ro.forward(*(_t(a, cuda) for a in us))
    g = ro.backward(*[a - _t(t, cuda) for a, t in zip(fin, ustar)])
    for a, c in zip(x, g):
        np.testing.assert_allclose(_np(a.grad), _np(c), rtol=0, atol=1e-5 * float(torch.abs(c).max()))


def test_rollout_96_ten_steps(cuda):
    """The 96^3 10-step rollout: FP32 and mixed-precision gradients against the FP64 form's."""
    import mpp
    from mpp.rollout import Rollout

    b, us, ustar = _rollout_case(96, 10, 5496)
    grads = {}
    for prec in ("fp64", "fp32", "fp16"):
        s = mpp.FlipBasin.from_scene(b, tol=1e-11 if prec == "fp64" else 1e-6, maxiter=300, precision=prec,
                                     graph=True)
        ro = Rollout(s, 10, 0.02)
        fin = ro.forward(*(_t(a, cuda) for a in us))
        g = ro.backward(*[a - _t(t, cuda) for a, t in zip(fin, ustar)])
        grads[prec] = np.concatenate([_np(a).astype(np.float64) for a in g])
        assert np.isfinite(grads[prec]).all()
    ref = grads["fp64"]
    for prec in ("fp32", "fp16"):
        assert np.linalg.norm(grads[prec] - ref) / np.linalg.norm(ref) <= 1e-3, prec
