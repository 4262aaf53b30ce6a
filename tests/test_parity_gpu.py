"""Parity of libmpp's CUDA kernels with the CPU oracle, through the C ABI.

Elementwise passes (rhs, diagonal, operator, V-cycle, gradient) are compared bit for
bit in FP32: the kernels follow the reference's operation order and the library is
built without FMA contraction. Whole solves differ only in the order of the dot
products' sums, so they are compared by the tolerance the projection is specified to:
pressure relative L2 difference <= 1e-4 and the same divergence at the same residual.
"""
import warnings

import numpy as np
import pytest

import oracle
from mpp import scene

pytestmark = pytest.mark.gpu

PRESSURE_RTOL = 1e-4  # pressure relative L2 difference, FP32 GPU vs FP32 oracle


def _t(a, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _np(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def basins():
    return {n: scene.box_basin(n, seed=1000 + n) for n in (16, 32, 64)}


def _projector(grid, **kw):
    import mpp

    return mpp.Projector(grid, **kw)


@pytest.mark.parametrize("n", [16, 32, 64])
def test_diag_rhs_bitexact(cuda, basins, n):
    b = basins[n]
    p = _projector(b.grid)
    types, phi = _t(b.types, cuda), _t(b.phi, cuda)
    d = _np(p.diag(types, phi))
    np.testing.assert_array_equal(d, oracle.diag(b.grid, b.types, b.phi))
    rhs = _np(p.rhs(_t(b.u, cuda), _t(b.v, cuda), _t(b.w, cuda), types, gamma=0.0123))
    np.testing.assert_array_equal(rhs, oracle.rhs(b.grid, b.u, b.v, b.w, b.types, np.float32(0.0123)))


@pytest.mark.parametrize("n", [16, 32, 64])
def test_apply_bitexact(cuda, basins, n):
    b = basins[n]
    p = _projector(b.grid)
    x = scene.uniform(7, 99, b.grid.ncells)
    y = _np(p.apply(_t(x, cuda), _t(b.types, cuda), _t(b.phi, cuda)))
    d = oracle.diag(b.grid, b.types, b.phi)
    np.testing.assert_array_equal(y, oracle.apply(b.grid, x, b.types, d))


@pytest.mark.parametrize("n", [16, 32, 64])
def test_vcycle_bitexact(cuda, basins, n):
    b = basins[n]
    p = _projector(b.grid)
    r = scene.uniform(11, 5, b.grid.ncells) * (b.types == scene.LIQUID)
    z = _np(p.vcycle(_t(r, cuda), _t(b.types, cuda), _t(b.phi, cuda)))
    d = oracle.diag(b.grid, b.types, b.phi)
    zo = oracle.vcycle(b.grid, r, b.types, d)
    np.testing.assert_array_equal(z, zo)


def test_gradient_bitexact(cuda, basins):
    b = basins[32]
    P = scene.uniform(3, 3, b.grid.ncells) * (b.types == scene.LIQUID)
    p = _projector(b.grid)
    u, v, w = _t(b.u, cuda), _t(b.v, cuda), _t(b.w, cuda)
    fu, fv, fw = (_t(np.zeros(a.size, np.uint8), cuda) for a in (b.u, b.v, b.w))
    p.gradient(u, v, w, fu, fv, fw, _t(P.astype(np.float32), cuda), _t(b.types, cuda), _t(b.phi, cuda))
    ref = oracle.gradient(b.grid, b.u, b.v, b.w, P.astype(np.float32), b.types, b.phi)
    for got, want in zip((u, v, w, fu, fv, fw), ref):
        np.testing.assert_array_equal(_np(got), want)


@pytest.mark.parametrize("n", [32, 64])
def test_volume(cuda, basins, n):
    b = basins[n]
    p = _projector(b.grid)
    got = p.volume(_t(b.phi, cuda))
    want = oracle.volume(b.grid, b.phi)
    assert abs(got - want) <= 1e-6 * abs(want)


@pytest.mark.parametrize("n,tol", [(32, 1e-4), (64, 1e-4), (64, 1e-6)])
@pytest.mark.parametrize("graph", [False, True])
def test_pressure_fp32_matches_oracle(cuda, basins, n, tol, graph):
    b = basins[n]
    bvec = oracle.rhs(b.grid, b.u, b.v, b.w, b.types, np.float32(0.0))
    P0 = np.zeros(b.grid.ncells, np.float32)
    Po, info = oracle.pressure(b.grid, P0, bvec, b.types, b.phi, tol=tol, maxiter=100)
    p = _projector(b.grid, tol=tol, maxiter=100, graph=graph)
    P = _t(P0, cuda)
    res = p.pressure(P, _t(bvec, cuda), _t(b.types, cuda), _t(b.phi, cuda))
    assert res.status == 0
    assert abs(res.iterations - info.iterations) <= 1
    Pg = _np(P)
    rel = np.linalg.norm(Pg - Po) / np.linalg.norm(Po)
    assert rel <= PRESSURE_RTOL, rel
    assert res.true_rel_residual <= 2 * tol


def _div_liquid(grid, u, v, w, types):
    n1, n2, n3 = grid.n
    U = u.reshape(n3, n2, n1 + 1)
    V = v.reshape(n3, n2 + 1, n1)
    W = w.reshape(n3 + 1, n2, n1)
    div = (U[:, :, 1:] - U[:, :, :-1]) + (V[:, 1:, :] - V[:, :-1, :]) + (W[1:, :, :] - W[:-1, :, :])
    return div.reshape(-1)[types == scene.LIQUID]


@pytest.mark.parametrize("graph", [False, True])
def test_project_fp32_matches_oracle(cuda, basins, graph):
    import mpp

    b = basins[64]
    vol0 = oracle.volume(b.grid, b.phi) * 1.002  # a little volume lost: gamma != 0
    ref = oracle.project(b, volume0=vol0, dt=1 / 48, tol=1e-6, maxiter=100)
    s = mpp.FlipBasin.from_scene(b, tol=1e-6, maxiter=100, graph=graph)
    s.volume0 = vol0
    mpp.project(s, 1 / 48)
    assert abs(s.last.gamma - ref["info"].gamma) <= 1e-6 * max(1.0, abs(ref["info"].gamma))
    assert abs(s.iterations[-1] - ref["info"].iterations) <= 1
    P = _np(s.P)
    assert np.linalg.norm(P - ref["P"]) / np.linalg.norm(ref["P"]) <= PRESSURE_RTOL
    np.testing.assert_array_equal(P[b.types != scene.LIQUID], 0.0)
    for got, want in zip((s.fu, s.fv, s.fw), (ref["fu"], ref["fv"], ref["fw"])):
        np.testing.assert_array_equal(_np(got), want)
    dg = np.abs(_div_liquid(b.grid, _np(s.u), _np(s.v), _np(s.w), b.types)).max()
    do = np.abs(_div_liquid(b.grid, ref["u"], ref["v"], ref["w"], b.types)).max()
    d0 = np.abs(_div_liquid(b.grid, b.u, b.v, b.w, b.types)).max()
    assert dg < 1e-3 * d0 + 2 * b.grid.dx * abs(s.last.gamma)
    assert dg <= 2 * do + 1e-6 * d0


def test_graph_equals_host_loop(cuda, basins):
    """The graph's device-side loop runs the same kernels in the same order: same bits."""
    b = basins[32]
    bvec = _t(oracle.rhs(b.grid, b.u, b.v, b.w, b.types, np.float32(0.0)), cuda)
    out = []
    for graph in (False, True):
        p = _projector(b.grid, tol=1e-6, maxiter=100, graph=graph)
        P = _t(np.zeros(b.grid.ncells, np.float32), cuda)
        res = p.pressure(P, bvec, _t(b.types, cuda), _t(b.phi, cuda))
        out.append((_np(P), res.iterations))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]


def test_fp64_matches_oracle(cuda, basins):
    b = basins[32]
    bvec = oracle.rhs(b.grid, b.u, b.v, b.w, b.types, np.float32(0.0))
    Po, info = oracle.pressure(b.grid, np.zeros(b.grid.ncells), bvec.astype(np.float64), b.types, b.phi, tol=1e-12,
                               maxiter=200, prec=64)
    p = _projector(b.grid, tol=1e-12, maxiter=200, precision="fp64")
    P = _t(np.zeros(b.grid.ncells, np.float32), cuda)
    res = p.pressure(P, _t(bvec, cuda), _t(b.types, cuda), _t(b.phi, cuda))
    assert res.status == 0
    P64 = p.solution_f64()
    assert np.linalg.norm(P64 - Po) / np.linalg.norm(Po) <= 1e-9


@pytest.mark.parametrize("prec", ["fp16", "bf16"])
def test_mixed_converges(cuda, basins, prec):
    b = basins[64]
    bvec = oracle.rhs(b.grid, b.u, b.v, b.w, b.types, np.float32(0.0))
    Pe, _ = oracle.pressure(b.grid, np.zeros(b.grid.ncells), bvec.astype(np.float64), b.types, b.phi, tol=1e-12,
                            maxiter=200, prec=64)
    p = _projector(b.grid, tol=1e-6, maxiter=100, precision=prec, graph=True)
    P = _t(np.zeros(b.grid.ncells, np.float32), cuda)
    res = p.pressure(P, _t(bvec, cuda), _t(b.types, cuda), _t(b.phi, cuda))
    assert res.status == 0, res.as_dict()
    assert res.true_rel_residual <= 2e-6
    err = np.linalg.norm(_np(P) - Pe) / np.linalg.norm(Pe)
    assert err <= 1e-4


@pytest.mark.parametrize("name", ["box16", "box32", "box32_gamma", "box16x16x32"])
@pytest.mark.parametrize("prec,tol,bound", [("fp64", 1e-12, 1e-9), ("fp32", 1e-6, 1e-4), ("fp16", 1e-6, 1e-4),
                                            ("bf16", 1e-6, 1e-4)])
def test_golden_exact_solution(cuda, name, prec, tol, bound):
    """Every form against the direct solve of the reference's equations (tests/golden)."""
    import os
    import sys

    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, gold)
    import make_golden

    kw, gamma = make_golden.CASES[name]
    basin = scene.box_basin(**kw)
    fx = np.load(os.path.join(gold, f"{name}.npz"))
    p = _projector(basin.grid, tol=tol, maxiter=300, precision=prec, graph=True)
    P = _t(np.zeros(basin.grid.ncells, np.float32), cuda)
    res = p.pressure(P, _t(fx["b"].astype(np.float32), cuda), _t(basin.types, cuda), _t(basin.phi, cuda))
    assert res.status == 0, res.as_dict()
    got = p.solution_f64() if prec == "fp64" else _np(P).astype(np.float64)
    # FP64 solves the FP32-rounded rhs: compare against the exact solution of that rhs
    exact = fx["P"]
    if prec == "fp64":
        b32 = fx["b"].astype(np.float32).astype(np.float64)
        P32, _ = oracle.pressure(basin.grid, np.zeros(basin.grid.ncells), b32, basin.types, basin.phi, tol=1e-13,
                                 maxiter=400, prec=64)
        exact = P32
    assert np.linalg.norm(got - exact) / np.linalg.norm(exact) <= bound


def test_not_converged_warns(cuda, basins):
    import mpp

    b = basins[32]
    s = mpp.FlipBasin.from_scene(b, tol=1e-8, maxiter=1)
    with warnings.catch_warnings(record=True) as rec:
        warnings.simplefilter("always")
        mpp.project(s, 1 / 48)
    assert s.iterations == [1]
    assert any("did not converge" in str(r.message) for r in rec)


def test_nonfinite_raises(cuda, basins):
    import mpp

    b = basins[16].copy()
    n1, n2, _ = b.grid.n
    c = int(np.flatnonzero(b.types == scene.LIQUID)[0])
    i, j, k = c % n1, (c // n1) % n2, c // (n1 * n2)
    b.u[i + 1 + (n1 + 1) * (j + n2 * k)] = np.nan  # the high-x face of a liquid cell
    s = mpp.FlipBasin.from_scene(b)
    with pytest.raises(RuntimeError, match="Nonfinite pressure"):
        mpp.project(s, 1 / 48)


def test_warm_start_and_zero_rhs(cuda, basins):
    """pressure! returns 0 when |b| = 0 or the warm start already meets tol."""
    b = basins[16]
    p = _projector(b.grid)
    zero = _t(np.zeros(b.grid.ncells, np.float32), cuda)
    P = _t(np.zeros(b.grid.ncells, np.float32), cuda)
    res = p.pressure(P, zero, _t(b.types, cuda), _t(b.phi, cuda))
    assert res.iterations == 0 and res.status == 0
    bvec = _t(oracle.rhs(b.grid, b.u, b.v, b.w, b.types, np.float32(0.0)), cuda)
    res = p.pressure(P, bvec, _t(b.types, cuda), _t(b.phi, cuda))
    assert res.iterations > 0
    res2 = p.pressure(P, bvec, _t(b.types, cuda), _t(b.phi, cuda))
    assert res2.iterations == 0
