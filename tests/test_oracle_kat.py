"""The oracle pinned: golden exact solutions, known-answer problems, algebraic properties.

The reference's test suite holds no values for the projection (parity unpinned), so the
oracle is checked against the reference's equations solved independently
(tests/golden/, scipy sparse LU), against closed-form answers, and for the properties
its algorithm guarantees (a symmetric operator, a symmetric positive V-cycle, a
divergence-free result).
"""
import os

import numpy as np
import pytest

import oracle
from mpp import scene

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _golden_cases():
    import sys

    sys.path.insert(0, GOLDEN)
    import make_golden

    return make_golden


@pytest.mark.parametrize("name", ["box16", "box32", "box32_gamma", "box16x16x32"])
def test_oracle_matches_golden_exact_solution(name):
    mg = _golden_cases()
    kw, gamma = mg.CASES[name]
    basin = scene.box_basin(**kw)
    fx = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    assert str(fx["digest"]) == mg.scene_digest(basin), "the scene generator changed"
    # the rhs: rhs_kernel! restated
    b64 = oracle.rhs(basin.grid, basin.u, basin.v, basin.w, basin.types, gamma, prec=64)
    np.testing.assert_allclose(b64, fx["b"], rtol=0, atol=1e-15)
    # FP64 PCG to 1e-12 against the direct solve
    P64, info = oracle.pressure(basin.grid, np.zeros(basin.grid.ncells), fx["b"], basin.types, basin.phi, tol=1e-12,
                                maxiter=300, prec=64)
    assert info.converged
    rel = np.linalg.norm(P64 - fx["P"]) / np.linalg.norm(fx["P"])
    assert rel < 1e-9, rel
    # FP32, the reference's arithmetic, to 1e-6
    b32 = oracle.rhs(basin.grid, basin.u, basin.v, basin.w, basin.types, np.float32(gamma))
    P32, info = oracle.pressure(basin.grid, np.zeros(basin.grid.ncells, np.float32), b32, basin.types, basin.phi,
                                tol=1e-6, maxiter=100)
    assert info.converged
    assert np.linalg.norm(P32 - fx["P"]) / np.linalg.norm(fx["P"]) < 1e-4


def _grid(n, levels):
    return scene.Grid(lo=(0.0, 0.0, 0.0), dx=0.1, n=n, radius=1e9, floor=-1e9, levels=levels)


def test_single_liquid_cell_under_air():
    """One LIQUID cell, AIR above, walls elsewhere: diag = 1/theta, P = b theta."""
    n = (2, 2, 4)
    g = _grid(n, 2)
    types = np.zeros(16, np.uint8)
    phi = np.ones(16, np.float32)
    c = 0 + 2 * (0 + 2 * 1)  # cell (0,0,1)
    a = 0 + 2 * (0 + 2 * 2)  # cell (0,0,2) above it
    types[c], types[a] = scene.LIQUID, scene.AIR
    phi[c], phi[a] = -0.03, 0.07  # theta = 0.03 / 0.1 = 0.3
    d = oracle.diag(g, types, phi, prec=64)
    assert d[c] == pytest.approx(1 / 0.3, rel=1e-6)
    b = np.zeros(16)
    b[c] = 0.6
    P, info = oracle.pressure(g, np.zeros(16), b, types, phi, tol=1e-14, maxiter=50, prec=64)
    assert P[c] == pytest.approx(0.6 * 0.3, rel=1e-6)
    assert np.count_nonzero(P) == 1


def test_water_column_closed_form():
    """A 1-D column of LIQUID cells over a wall, AIR on top: the reference's operator is
    the tridiagonal (1, 2, ..., 2, 1 + 1/theta) Neumann-Dirichlet matrix."""
    n = (2, 2, 8)
    g = _grid(n, 2)
    types = np.zeros(32, np.uint8)
    phi = np.full(32, 1.0, np.float32)
    depth = 5
    col = [0 + 2 * (0 + 2 * k) for k in range(8)]
    for k in range(8):
        types[col[k]] = scene.LIQUID if k < depth else scene.AIR
        phi[col[k]] = (k + 0.5) * 0.1 - 0.52  # surface between k=4 (-0.07) and k=5 (+0.03)
    theta = 0.07 / 0.1
    A = np.zeros((depth, depth))
    for k in range(depth):
        if k > 0:
            A[k, k - 1] = -1
            A[k, k] += 1
        if k < depth - 1:
            A[k, k + 1] = -1
            A[k, k] += 1
    A[depth - 1, depth - 1] += 1 / theta
    rhs = np.linspace(0.1, 0.5, depth)
    exact = np.linalg.solve(A, rhs)
    b = np.zeros(32)
    b[col[:depth]] = rhs
    P, info = oracle.pressure(g, np.zeros(32), b, types, phi, tol=1e-14, maxiter=100, prec=64)
    # phi is Float32 (as the reference's), so theta carries a ~1e-8 relative rounding
    np.testing.assert_allclose(P[col[:depth]], exact, rtol=1e-6)


@pytest.fixture(scope="module")
def b24():
    return scene.box_basin(24, seed=99, height=0.5)


def test_operator_symmetric(b24):
    g = b24.grid
    d = oracle.diag(g, b24.types, b24.phi, prec=64)
    live = b24.types == scene.LIQUID
    x = scene.uniform(1, 1, g.ncells).astype(np.float64) * live
    y = scene.uniform(2, 2, g.ncells).astype(np.float64) * live
    ax = oracle.apply(g, x, b24.types, d, prec=64)
    ay = oracle.apply(g, y, b24.types, d, prec=64)
    assert abs(ax @ y - x @ ay) <= 1e-12 * abs(ax @ y)
    assert x @ ax > 0


@pytest.mark.parametrize("sweeps,sweeps_coarse,coarse", [(2, 0, 40), (5, 6, 10), (1, 3, 4)])
def test_vcycle_symmetric_positive(b24, sweeps, sweeps_coarse, coarse):
    """The V-cycle reverses its colour order on the way up (src/flip.jl:996) and solves the
    coarsest level symmetrically (:945), so M is symmetric positive definite; that holds
    level by level, so for any per-level sweep counts (the autotuner's) too."""
    g = b24.grid
    d = oracle.diag(g, b24.types, b24.phi, prec=64)
    live = b24.types == scene.LIQUID
    x = scene.uniform(3, 3, g.ncells).astype(np.float64) * live
    y = scene.uniform(4, 4, g.ncells).astype(np.float64) * live
    kw = dict(sweeps=sweeps, sweeps_coarse=sweeps_coarse, coarse=coarse, prec=64)
    mx = oracle.vcycle(g, x, b24.types, d, **kw)
    my = oracle.vcycle(g, y, b24.types, d, **kw)
    assert abs(mx @ y - x @ my) <= 1e-10 * abs(mx @ y)
    assert mx @ x > 0 and my @ y > 0


def test_vcycle_coarse_sweeps_default_is_the_reference(b24):
    """A coarser-level count of 0, or equal to the fine one, is the reference's one `sweeps`;
    a different one changes the result once the grid has a level between fine and coarsest."""
    g = b24.grid
    d = oracle.diag(g, b24.types, b24.phi)
    r = scene.uniform(5, 5, g.ncells) * (b24.types == scene.LIQUID)
    base = oracle.vcycle(g, r, b24.types, d, sweeps=3)
    np.testing.assert_array_equal(oracle.vcycle(g, r, b24.types, d, sweeps=3, sweeps_coarse=3), base)
    assert g.levels >= 3
    assert not np.array_equal(oracle.vcycle(g, r, b24.types, d, sweeps=3, sweeps_coarse=1), base)


def test_projection_removes_divergence(b24):
    vol0 = oracle.volume(b24.grid, b24.phi, prec=64)  # no volume loss: gamma = 0
    out = oracle.project(b24, volume0=vol0, tol=1e-12, maxiter=300, prec=64)
    n1, n2, n3 = b24.grid.n
    live = b24.types == scene.LIQUID

    def div(u, v, w):
        U, V, W = u.reshape(n3, n2, n1 + 1), v.reshape(n3, n2 + 1, n1), w.reshape(n3 + 1, n2, n1)
        d = (U[:, :, 1:] - U[:, :, :-1]) + (V[:, 1:, :] - V[:, :-1, :]) + (W[1:, :, :] - W[:-1, :, :])
        return d.reshape(-1)[live]

    before = np.abs(div(b24.u, b24.v, b24.w)).max()
    after = np.abs(div(out["u"], out["v"], out["w"])).max()
    assert after < 1e-9 * before
    # the valid flags are exactly the faces with a LIQUID side and no SOLID one
    assert out["fu"].sum() > 0 and set(np.unique(out["fu"])) <= {0, 1}


def test_fp32_oracle_iterations_close_to_fp64(b24):
    vol0 = oracle.volume(b24.grid, b24.phi)
    o32 = oracle.project(b24, volume0=vol0, tol=1e-6, maxiter=100)
    o64 = oracle.project(b24, volume0=vol0, tol=1e-6, maxiter=100, prec=64)
    assert abs(o32["info"].iterations - o64["info"].iterations) <= 1
    assert np.linalg.norm(o32["P"] - o64["P"]) / np.linalg.norm(o64["P"]) < 1e-4


def test_volume_gamma_clamp(b24):
    """project!'s gamma = clamp(loss / recover, -0.01/dt, 0.01/dt) (src/flip.jl:1146-1147)."""
    vol = oracle.volume(b24.grid, b24.phi)
    out = oracle.project(b24, volume0=vol * 2.0, dt=0.5, recover=0.5, tol=1e-3)
    assert out["info"].gamma == pytest.approx(0.01 / 0.5, rel=1e-6)
    out = oracle.project(b24, volume0=vol * 1.001, dt=0.5, recover=0.5, tol=1e-3)
    loss = np.float32((np.float32(vol * 1.001) - np.float32(vol)) / np.float32(vol * 1.001))
    assert out["info"].gamma == pytest.approx(float(loss) / 0.5, rel=1e-4)
