"""The FGMRES fallback (src/fgmres.jl:26-110) through the C ABI.

CG is held to a few iterations (``cg_maxiter_with_fallback``) so that it misses the
tolerance and the flexible GMRES takes over; the result must meet the same true-residual
tolerance and agree with the FP64 oracle's solution of the same equations.
"""
import warnings

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


@pytest.fixture(scope="module")
def basin64():
    b = scene.box_basin(64, seed=1064)
    bvec = oracle.rhs(b.grid, b.u, b.v, b.w, b.types, np.float32(0.0))
    Pe, _ = oracle.pressure(b.grid, np.zeros(b.grid.ncells), bvec.astype(np.float64), b.types, b.phi, tol=1e-12,
                            maxiter=200, prec=64)
    return b, bvec, Pe


def _rel_residual(b, bvec, P, prec):
    d = oracle.diag(b.grid, b.types, b.phi, prec=64) if prec == "fp64" else oracle.diag(b.grid, b.types, b.phi)
    r = bvec.astype(np.float64) - oracle.apply(b.grid, P, b.types, d.astype(np.float64), prec=64)
    r[b.types != scene.LIQUID] = 0.0
    return np.linalg.norm(r) / np.linalg.norm(bvec.astype(np.float64))


def _solve(b, bvec, cuda, P0=None, **kw):
    import mpp

    p = mpp.Projector(b.grid, **kw)
    P = _t(np.zeros(b.grid.ncells, np.float32) if P0 is None else P0, cuda)
    res = p.pressure(P, _t(bvec, cuda), _t(b.types, cuda), _t(b.phi, cuda))
    return p, P, res


@pytest.mark.parametrize("prec,tol,bound", [("fp32", 1e-5, 5e-3), ("fp16", 1e-5, 5e-3), ("bf16", 1e-5, 5e-3),
                                            ("fp64", 1e-10, 5e-8)])
@pytest.mark.parametrize("restart", [4, 8])
def test_fgmres_converges_after_cg(cuda, basin64, prec, tol, bound, restart):
    b, bvec, Pe = basin64
    p, P, res = _solve(b, bvec, cuda, tol=tol, maxiter=100, precision=prec, graph=True, fallback=True,
                       restart=restart, cg_maxiter_with_fallback=2)
    assert res.status == 0, res.as_dict()
    assert res.iterations == 2
    assert res.fallback_used == 1 and res.fallback_iterations > 0
    assert res.true_rel_residual <= tol
    got = p.solution_f64() if prec == "fp64" else _np(P).astype(np.float64)
    # the contract is the true residual (src/fgmres.jl:90), recomputed here in FP64 on the
    # equations the form solves (FP32 diagonal except in the FP64 form)
    assert _rel_residual(b, bvec, got, prec) <= tol * 1.05
    # GMRES minimises the residual, not the energy norm: the error is bounded by the
    # operator's conditioning (~n^2) times tol
    assert np.linalg.norm(got - Pe) / np.linalg.norm(Pe) <= bound
    np.testing.assert_array_equal(_np(P)[b.types != scene.LIQUID], 0.0)


def test_fgmres_tight_fp32(cuda, basin64):
    b, bvec, Pe = basin64
    _, P, res = _solve(b, bvec, cuda, tol=1e-6, maxiter=100, graph=True, fallback=True, cg_maxiter_with_fallback=1)
    assert res.status == 0 and res.fallback_used == 1, res.as_dict()
    assert res.true_rel_residual <= 1e-6
    assert _rel_residual(b, bvec, _np(P).astype(np.float64), "fp32") <= 1.05e-6
    assert np.linalg.norm(_np(P) - Pe) / np.linalg.norm(Pe) <= 5e-4


def test_no_fallback_when_cg_converges(cuda, basin64):
    """CG that meets tol on its true residual is kept: same bits as without the fallback."""
    b, bvec, _ = basin64
    _, P1, r1 = _solve(b, bvec, cuda, tol=1e-6, maxiter=100, graph=True)
    _, P2, r2 = _solve(b, bvec, cuda, tol=1e-6, maxiter=100, graph=True, fallback=True)
    assert r2.fallback_used == 0 and r2.fallback_iterations == 0
    assert r1.iterations == r2.iterations
    np.testing.assert_array_equal(_np(P1), _np(P2))


def test_graph_and_host_loop_same_bits(cuda, basin64):
    b, bvec, _ = basin64
    out = []
    for graph in (False, True):
        _, P, res = _solve(b, bvec, cuda, tol=1e-5, maxiter=100, graph=graph, fallback=True,
                           cg_maxiter_with_fallback=3)
        assert res.fallback_used == 1
        out.append((_np(P), res.fallback_iterations))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]


def test_diverged_start_is_zeroed(cuda, basin64):
    """A warm start whose residual is above 2|b| is dropped before FGMRES (src/fgmres.jl:109)."""
    b, bvec, Pe = basin64
    P0 = (scene.uniform(5, 77, b.grid.ncells) * 1e4 * (b.types == scene.LIQUID)).astype(np.float32)
    _, P, res = _solve(b, bvec, cuda, P0=P0, tol=1e-5, maxiter=100, graph=True, fallback=True,
                       cg_maxiter_with_fallback=1)
    assert res.status == 0 and res.fallback_used == 1, res.as_dict()
    assert _rel_residual(b, bvec, _np(P).astype(np.float64), "fp32") <= 1.05e-5


def test_fallback_not_converged_raises(cuda, basin64):
    """FGMRES that misses tol is an error, not a warning (src/fgmres.jl:90)."""
    import mpp

    b, bvec, _ = basin64
    _, _, res = _solve(b, bvec, cuda, tol=1e-9, maxiter=100, fallback=True, cg_maxiter_with_fallback=1,
                       fallback_maxiter=2)
    assert res.status == 1 and res.fallback_used == 1 and res.fallback_iterations == 2
    s = mpp.FlipBasin.from_scene(b, tol=1e-9, maxiter=100, fallback=True, cg_maxiter_with_fallback=1,
                                 fallback_maxiter=2)
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        with pytest.raises(RuntimeError, match="Pressure did not converge"):
            mpp.project(s, 1 / 48)


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_project_with_fallback(cuda, basin64, prec):
    """project! with the fallback: the gradient update follows FGMRES's pressure."""
    import mpp

    b, _, _ = basin64
    vol0 = oracle.volume(b.grid, b.phi) * 1.002
    ref = oracle.project(b, volume0=vol0, dt=1 / 48, tol=1e-6, maxiter=100)
    s = mpp.FlipBasin.from_scene(b, tol=1e-5, maxiter=100, precision=prec, graph=True, fallback=True,
                                 cg_maxiter_with_fallback=2)
    s.volume0 = vol0
    mpp.project(s, 1 / 48)
    assert s.last.fallback_used == 1
    P = _np(s.P)
    assert np.linalg.norm(P - ref["P"]) / np.linalg.norm(ref["P"]) <= 5e-3
    for got, want in zip((s.fu, s.fv, s.fw), (ref["fu"], ref["fv"], ref["fw"])):
        np.testing.assert_array_equal(_np(got), want)
    # the velocity update is the gradient of that pressure: divergence at tol on liquid cells
    n1, n2, n3 = b.grid.n
    U = _np(s.u).reshape(n3, n2, n1 + 1)
    V = _np(s.v).reshape(n3, n2 + 1, n1)
    W = _np(s.w).reshape(n3 + 1, n2, n1)
    div = ((U[:, :, 1:] - U[:, :, :-1]) + (V[:, 1:, :] - V[:, :-1, :]) + (W[1:, :, :] - W[:-1, :, :])).reshape(-1)
    U0 = b.u.reshape(n3, n2, n1 + 1)
    V0 = b.v.reshape(n3, n2 + 1, n1)
    W0 = b.w.reshape(n3 + 1, n2, n1)
    div0 = ((U0[:, :, 1:] - U0[:, :, :-1]) + (V0[:, 1:, :] - V0[:, :-1, :]) + (W0[1:, :, :] - W0[:-1, :, :])).reshape(-1)
    liq = b.types == scene.LIQUID
    assert np.abs(div[liq]).max() < 1e-2 * np.abs(div0[liq]).max() + 2 * b.grid.dx * abs(s.last.gamma)
