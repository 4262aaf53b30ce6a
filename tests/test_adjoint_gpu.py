"""The adjoint of project! on the GPU (mpp_project_vjp) against the oracle and against
FP64 central differences of the oracle's FP64 forward.

Loss 1/2 |P(u) - u*|^2 with u and u* uniform[-1, 1] m/s. The map is affine in u, so
central differences are exact up to rounding and solve tolerance.
"""
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


def _setup(n, seed):
    b = scene.box_basin(n, seed=seed)
    rng = np.random.default_rng(seed)
    ustar = [rng.uniform(-1, 1, a.size).astype(np.float32) for a in (b.u, b.v, b.w)]
    return b, rng, ustar


@pytest.mark.parametrize("n", [16, 32, 64])
def test_vjp_passes_bitexact(cuda, n):
    import mpp

    b, rng, _ = _setup(n, 3000 + n)
    gs = [rng.uniform(-1, 1, a.size).astype(np.float32) for a in (b.u, b.v, b.w)]
    mu = (rng.uniform(-1, 1, b.grid.ncells) * (b.types == scene.LIQUID)).astype(np.float32)
    p = mpp.Projector(b.grid)
    T, F = _t(b.types, cuda), _t(b.phi, cuda)
    beta = _np(p.vjp_rhs(*(_t(a, cuda) for a in gs), T, F))
    np.testing.assert_array_equal(beta, oracle.vjp_rhs(b.grid, *gs, b.types, b.phi))
    outs = p.vjp_faces(*(_t(a, cuda) for a in gs), _t(mu, cuda), T)
    for got, want in zip(outs, oracle.vjp_faces(b.grid, *gs, mu, b.types)):
        np.testing.assert_array_equal(_np(got), want)


def _gpu_grad(b, ustar, cuda, prec, tol, **kw):
    """Forward project! on the GPU, cotangent P(u) - u*, then the GPU adjoint."""
    import mpp

    s = mpp.FlipBasin.from_scene(b, tol=tol, maxiter=300, precision=prec, graph=True, **kw)
    s.volume0 = oracle.volume(b.grid, b.phi) * 1.002
    mpp.project(s, 1 / 48)
    cot = [a - _t(us, cuda) for a, us in zip((s.u, s.v, s.w), ustar)]
    mpp.project_vjp(s, *cot)
    return [_np(a).astype(np.float64) for a in cot], s


def test_fp64_adjoint_matches_central_differences(cuda):
    """FP64 form: gradient . d against FP64 central differences, 8 random directions, 32^3."""
    b, rng, ustar = _setup(32, 3032)
    g = b.grid
    grad, _ = _gpu_grad(b, ustar, cuda, "fp64", 1e-12)
    vol0 = oracle.volume(g, b.phi) * 1.002
    u0 = [a.astype(np.float64) for a in (b.u, b.v, b.w)]

    def loss(us):
        bb = b.copy()
        bb.u, bb.v, bb.w = us
        r = oracle.project(bb, volume0=vol0, dt=1 / 48, tol=1e-13, maxiter=400, prec=64)
        return 0.5 * sum(((r[k] - s.astype(np.float64)) ** 2).sum() for k, s in zip("uvw", ustar))

    h = 1e-3
    fds, ans = [], []
    for _ in range(8):
        d = [rng.uniform(-1, 1, a.size) for a in u0]
        fds.append((loss([a + h * e for a, e in zip(u0, d)]) - loss([a - h * e for a, e in zip(u0, d)])) / (2 * h))
        ans.append(sum((gg * e).sum() for gg, e in zip(grad, d)))
    fds, ans = np.array(fds), np.array(ans)
    # The arrays crossing the ABI are Float32 (as the reference's), so the cotangent and
    # the gradient carry a rounding of ~6e-8 per element; a direction whose derivative
    # happens to be small sees it amplified. The 8 directional derivatives as a vector
    # must agree to 1e-6, each one to 1e-5.
    assert np.linalg.norm(ans - fds) / np.linalg.norm(fds) <= 1e-6, (ans, fds)
    assert (np.abs(ans - fds) / np.abs(fds)).max() <= 1e-5, (ans, fds)


@pytest.mark.parametrize("n,prec,bound", [(32, "fp32", 1e-4), (64, "fp32", 1e-4), (64, "fp16", 1e-4),
                                          (64, "bf16", 1e-4)])
def test_adjoint_matches_fp64_reference_gradient(cuda, n, prec, bound):
    """Every form's gradient against the oracle's FP64 adjoint of the same cotangent."""
    b, _, ustar = _setup(n, 3100 + n)
    grad, _ = _gpu_grad(b, ustar, cuda, prec, 1e-6)
    # the FP64 reference: FP64 forward and FP64 adjoint on the CPU
    vol0 = oracle.volume(b.grid, b.phi) * 1.002
    r = oracle.project(b, volume0=vol0, dt=1 / 48, tol=1e-13, maxiter=400, prec=64)
    cot = [r[k] - s.astype(np.float64) for k, s in zip("uvw", ustar)]
    ref = oracle.project_vjp(b, *cot, tol=1e-13, maxiter=400, prec=64)
    want = np.concatenate([ref["gu"], ref["gv"], ref["gw"]])
    got = np.concatenate(grad)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= bound


def test_adjoint_with_fallback(cuda):
    """The adjoint solve takes the same FGMRES fallback as the forward."""
    b, _, ustar = _setup(32, 3232)
    g1, _ = _gpu_grad(b, ustar, cuda, "fp32", 1e-6)
    g2, s = _gpu_grad(b, ustar, cuda, "fp32", 1e-6, fallback=True, cg_maxiter_with_fallback=2)
    assert s.last_vjp.fallback_used == 1
    a, c = np.concatenate(g1), np.concatenate(g2)
    assert np.linalg.norm(a - c) / np.linalg.norm(a) <= 1e-4


def test_autograd_function(cuda):
    """torch.autograd through ProjectFunction equals the explicit pullback."""
    import torch

    import mpp
    from mpp import adjoint

    b, _, ustar = _setup(32, 3332)
    s = mpp.FlipBasin.from_scene(b, tol=1e-6, maxiter=200)
    s.volume0 = oracle.volume(b.grid, b.phi) * 1.002
    u, v, w = (_t(a, cuda).requires_grad_(True) for a in (b.u, b.v, b.w))
    uo, vo, wo = adjoint.project(u, v, w, s, 1 / 48)
    loss = 0.5 * sum(((o - _t(t, cuda)) ** 2).sum() for o, t in zip((uo, vo, wo), ustar))
    loss.backward()
    # explicit pullback on a fresh basin
    grad, _ = _gpu_grad(b, ustar, cuda, "fp32", 1e-6)
    for a, gref in zip((u.grad, v.grad, w.grad), grad):
        np.testing.assert_allclose(_np(a), gref, rtol=0, atol=1e-5 * np.abs(gref).max())
    assert isinstance(loss, torch.Tensor)


def test_adjoint_128(cuda):
    """128^3 (the adjoint workload): FP32 and mixed gradients against the FP64 form's."""
    b, _, ustar = _setup(128, 3128)
    ref, _ = _gpu_grad(b, ustar, cuda, "fp64", 1e-11)
    want = np.concatenate(ref)
    for prec in ("fp32", "fp16"):
        got, _ = _gpu_grad(b, ustar, cuda, prec, 1e-6)
        assert np.linalg.norm(np.concatenate(got) - want) / np.linalg.norm(want) <= 1e-4
