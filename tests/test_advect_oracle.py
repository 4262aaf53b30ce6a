"""The oracle's advection adjoint and rollout adjoint against FP64 central differences.

The velocities are uniform[-1, 1] on every face (not walled), so no trajectory starts
exactly on a clamp boundary of the trilinear lookup, where the derivative is one-sided.
"""
import numpy as np
import pytest

import oracle
from mpp import scene


def _flow(g, seed, scale=1.0):
    return [(scene.uniform(seed, 20 + a, int(np.prod(g.face_shape(a)))) * scale).astype(np.float64) for a in range(3)]


def _fd(loss, x0, dirs, h):
    return np.array([(loss([a + h * e for a, e in zip(x0, d)]) - loss([a - h * e for a, e in zip(x0, d)])) / (2 * h)
                     for d in dirs])


@pytest.mark.parametrize("scale", [0.5, 3.0])  # 3 m/s: some nodes take 2 sub-steps
def test_advect_adjoint_matches_central_differences(scale):
    b = scene.box_basin(16, seed=4016)
    g = b.grid
    us = _flow(g, 41, scale)
    rng = np.random.default_rng(1)
    ustar = [rng.uniform(-1, 1, a.size) for a in us]
    dt = 0.02

    def loss(x):
        return 0.5 * sum(((a - s) ** 2).sum() for a, s in zip(oracle.advect_velocity(g, *x, dt, prec=64), ustar))

    cot = [a - s for a, s in zip(oracle.advect_velocity(g, *us, dt, prec=64), ustar)]
    grad = oracle.advect_velocity_vjp(g, *cot, *us, dt, prec=64)
    dirs = [[rng.uniform(-1, 1, a.size) for a in us] for _ in range(6)]
    fd = _fd(loss, us, dirs, 1e-6)
    an = np.array([sum((x * e).sum() for x, e in zip(grad, d)) for d in dirs])
    assert np.linalg.norm(an - fd) / np.linalg.norm(fd) <= 1e-6, (an, fd)


def test_advect_level_set_shape():
    b = scene.box_basin(16, seed=4017)
    g = b.grid
    us = _flow(g, 42)
    out = oracle.advect(g, b.phi, None, *us, 0.02)
    assert out.shape == (g.ncells,) and np.isfinite(out).all()
    # a zero flow leaves every array as it is, up to the rounding of the node positions
    z = [np.zeros_like(a, dtype=np.float32) for a in us]
    np.testing.assert_allclose(oracle.advect(g, b.phi, None, *z, 0.02), b.phi, rtol=0, atol=1e-5)


def test_rollout_adjoint_matches_central_differences():
    """3 steps of advect + project at 16^3, FP64: reverse pass against central differences."""
    b = scene.box_basin(16, seed=4018)
    g = b.grid
    us = _flow(g, 43)
    rng = np.random.default_rng(2)
    ustar = [rng.uniform(-1, 1, a.size) for a in us]
    dt, steps = 0.02, 3

    def loss(x):
        st = oracle.rollout(b, *x, steps, dt)
        return 0.5 * sum(((a - s) ** 2).sum() for a, s in zip(st[-1], ustar))

    st = oracle.rollout(b, *us, steps, dt)
    cot = [a - s for a, s in zip(st[-1], ustar)]
    grad = oracle.rollout_vjp(b, st, *cot, dt)
    dirs = [[rng.uniform(-1, 1, a.size) for a in us] for _ in range(4)]
    fd = _fd(loss, us, dirs, 1e-6)
    an = np.array([sum((x * e).sum() for x, e in zip(grad, d)) for d in dirs])
    assert np.linalg.norm(an - fd) / np.linalg.norm(fd) <= 1e-6, (an, fd)
