"""The oracle's adjoint of project! against FP64 central differences of its own forward.

project! is affine in the face velocities for fixed cell classes and level set, so the
loss 1/2 |P(u) - u*|^2 is quadratic and its central difference is exact up to rounding
and the solve tolerance: the adjoint must agree to far below 1e-6.
"""
import numpy as np
import pytest

import oracle
from mpp import scene


def _loss_and_fd(b, ustar, dirs, h=1e-3):
    g = b.grid
    vol0 = oracle.volume(g, b.phi) * 1.002
    u0 = [a.astype(np.float64) for a in (b.u, b.v, b.w)]

    def fwd(us):
        bb = b.copy()
        bb.u, bb.v, bb.w = us
        return oracle.project(bb, volume0=vol0, dt=1 / 48, tol=1e-13, maxiter=400, prec=64)

    def loss(us):
        r = fwd(us)
        return 0.5 * sum(((r[k] - s) ** 2).sum() for k, s in zip("uvw", ustar))

    r0 = fwd(u0)
    cot = [r0[k] - s for k, s in zip("uvw", ustar)]
    fds = []
    for d in dirs:
        lp = loss([a + h * e for a, e in zip(u0, d)])
        lm = loss([a - h * e for a, e in zip(u0, d)])
        fds.append((lp - lm) / (2 * h))
    return cot, np.array(fds)


@pytest.mark.parametrize("n,ndir", [(16, 8), (32, 8)])
def test_oracle_adjoint_matches_central_differences(n, ndir):
    b = scene.box_basin(n, seed=2000 + n)
    rng = np.random.default_rng(n)
    ustar = [rng.uniform(-1, 1, a.size) for a in (b.u, b.v, b.w)]
    dirs = [[rng.uniform(-1, 1, a.size) for a in (b.u, b.v, b.w)] for _ in range(ndir)]
    cot, fd = _loss_and_fd(b, ustar, dirs)
    adj = oracle.project_vjp(b, *cot, tol=1e-13, maxiter=400, prec=64)
    an = np.array([sum((g * e).sum() for g, e in zip((adj["gu"], adj["gv"], adj["gw"]), d)) for d in dirs])
    rel = np.abs(an - fd) / np.abs(fd)
    assert rel.max() <= 1e-9, rel


def test_oracle_vjp_passes_are_transposes():
    """<G^T g, P> = <g, G P> and <D^T mu, u> = <mu, D u> on the oracle's own passes."""
    b = scene.box_basin(16, seed=2016)
    g = b.grid
    rng = np.random.default_rng(3)
    liquid = b.types == scene.LIQUID
    P = rng.uniform(-1, 1, g.ncells) * liquid
    gs = [rng.uniform(-1, 1, a.size) for a in (b.u, b.v, b.w)]
    # G P through the oracle's gradient pass on zero faces: u_out = -G P
    zeros = [np.zeros(a.size) for a in (b.u, b.v, b.w)]
    bb = b.copy()
    bb.u, bb.v, bb.w = zeros
    flags = [np.zeros(a.size, np.uint8) for a in zeros]
    us = [z.copy() for z in zeros]
    oracle.lib().orc_gradient_f64(oracle.ctypes.byref(oracle._grid(g)), *(oracle._p(a) for a in us),
                                  *(oracle._p(f) for f in flags), oracle._p(P),
                                  oracle._p(np.ascontiguousarray(b.types)),
                                  oracle._p(np.ascontiguousarray(b.phi, dtype=np.float64)))
    GP = [-a * g.dx for a in us]  # dx G P
    beta = oracle.vjp_rhs(g, *gs, b.types, b.phi, prec=64)  # dx G^T g
    lhs = (beta * P).sum()
    rhs = sum((a * c).sum() for a, c in zip(gs, GP))
    assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs))
    # D^T: g_in - g = D^T mu; D u = -rhs/dx at gamma = 0
    mu = rng.uniform(-1, 1, g.ncells) * liquid
    outs = oracle.vjp_faces(g, *zeros, mu, b.types, prec=64)
    us = [rng.uniform(-1, 1, a.size) for a in (b.u, b.v, b.w)]
    Du = -oracle.rhs(g, *us, b.types, 0.0, prec=64) / g.dx
    lhs = sum((o * a).sum() for o, a in zip(outs, us))
    rhs = (mu * Du).sum()
    assert abs(lhs - rhs) <= 1e-10 * max(1.0, abs(lhs))
