"""The sparse basin's CPU oracle (oracle/sparse.c) pinned without the reference (which runs
on Julia and a Vulkan device, neither present here):

* the level-0 couplings and Dirichlet diagonal against a second restatement written here
  in numpy Float32 from src/sflip.jl:1324-1374 (celltype, finecoef_kernel!,
  finedirichlet_kernel!), bit for bit;
* algebraic properties of the composite operator (Losasso's coupling is symmetric and the
  operator positive definite on the unknowns; A 1 is the Dirichlet diagonal);
* the V-cycle's exact scaling (every operation of vcycle! scales exactly by a power of two);
* the projection's purpose: after project! the discrete divergence of the fine cells and
  the uncovered coarse cells (the right-hand side the next projection would see) is the
  solver's residual, which only holds when the gradient update, the face restriction and
  the coupling agree with each other.
"""
import numpy as np
import pytest

from mpp import sparse_scene as ss
from oracle import sparse as osp

SOLID, LIQUID, AIR = 0, 1, 2


@pytest.fixture(scope="module")
def scene():
    return ss.sparse_basin((4, 4, 4), seed=2101, warm=True)


def _unknowns(sc):
    fine = (sc.tf == LIQUID) & np.repeat(sc.where[:, 0] >= 0, 4096)
    nc = sc.grid.nc
    cov = np.zeros(nc, bool)
    for w in sc.where:
        if w[0] >= 0:
            cov[w[0] * 4:w[0] * 4 + 4, w[1] * 4:w[1] * 4 + 4, w[2] * 4:w[2] * 4 + 4] = True
    coarse = (sc.tc == LIQUID) & ~cov.reshape(-1, order="F")
    return fine, coarse


def _global_types(sc):
    """Each fine-resolution cell's (type, fine?) as celltype reads it (src/sflip.jl:1335-1342),
    on a dense array over the whole grid padded by one cell of SOLID."""
    nb, nf = sc.grid.nb, [16 * b for b in sc.grid.nb]
    tc = sc.tc.reshape(sc.grid.nc, order="F")
    t = np.repeat(np.repeat(np.repeat(tc, 4, 0), 4, 1), 4, 2)
    fine = np.zeros(nf, bool)
    phic = sc.phic.reshape(sc.grid.nc, order="F")
    phi = np.repeat(np.repeat(np.repeat(phic, 4, 0), 4, 1), 4, 2).astype(np.float32)
    for s, w in enumerate(sc.where):
        if w[0] < 0:
            continue
        blk = np.s_[w[0] * 16:w[0] * 16 + 16, w[1] * 16:w[1] * 16 + 16, w[2] * 16:w[2] * 16 + 16]
        t[blk] = sc.tf[s * 4096:(s + 1) * 4096].reshape(16, 16, 16).transpose(2, 1, 0)
        phi[blk] = sc.phif[s * 4096:(s + 1) * 4096].reshape(16, 16, 16).transpose(2, 1, 0)
        fine[blk] = True
    T = np.full([n + 2 for n in nf], SOLID, np.uint8)
    F = np.zeros([n + 2 for n in nf], bool)
    PH = np.zeros([n + 2 for n in nf], np.float32)
    T[1:-1, 1:-1, 1:-1], F[1:-1, 1:-1, 1:-1], PH[1:-1, 1:-1, 1:-1] = t, fine, phi
    # outside the grid: neighbourφ clamps to the edge coarse cell; only read for AIR, which
    # the SOLID padding never is
    return T, F, PH


def test_level0_coefficients_match_a_numpy_restatement(scene):
    sc = scene
    got = osp.coefficients(sc)
    T, F, PH = _global_types(sc)
    li = np.arange(4096)
    for a, key in ((0, "cuf"), (1, "cvf"), (2, "cwf")):
        want = np.zeros(sc.nslots * 4352, np.float32)
        f = np.arange(4352)
        if a == 0:
            i, j, k = f % 17, (f // 17) % 16, f // 272
        elif a == 1:
            i, j, k = f % 16, (f // 16) % 17, f // 272
        else:
            i, j, k = f % 16, (f // 16) % 16, f // 256
        e = np.eye(3, dtype=int)[a]
        for s, w in enumerate(sc.where):
            if w[0] < 0:
                continue
            I, J, K = w[0] * 16 + i + 1, w[1] * 16 + j + 1, w[2] * 16 + k + 1  # padded
            tp, fp = T[I, J, K], F[I, J, K]
            tm, fm = T[I - e[0], J - e[1], K - e[2]], F[I - e[0], J - e[1], K - e[2]]
            c = np.where((tp == LIQUID) & (tm == LIQUID), np.where(fp & fm, np.float32(1), np.float32(0.4)), 0)
            want[s * 4352:(s + 1) * 4352] = c
        assert np.array_equal(got[key].view(np.uint32), want.view(np.uint32)), key
    # finedirichlet_kernel!: the AIR neighbours' c / theta, in neighbour order +x,-x,+y,-y,+z,-z
    wantd = np.zeros(sc.nslots * 4096, np.float32)
    i, j, k = li % 16, (li // 16) % 16, li // 256
    nbs = ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))
    for s, w in enumerate(sc.where):
        if w[0] < 0:
            continue
        I, J, K = w[0] * 16 + i + 1, w[1] * 16 + j + 1, w[2] * 16 + k + 1
        pc = PH[I, J, K]
        d = np.zeros(4096, np.float32)
        liquid = T[I, J, K] == LIQUID
        for (dx, dy, dz) in nbs:
            tn, fn, pn = T[I + dx, J + dy, K + dz], F[I + dx, J + dy, K + dz], PH[I + dx, J + dy, K + dz]
            with np.errstate(divide="ignore", invalid="ignore"):
                th = (pc / (pc - pn)).astype(np.float32)
                th = np.where(th > 1, np.float32(1), np.where(th < np.float32(0.01), np.float32(0.01), th))
                term = (np.where(fn, np.float32(1), np.float32(0.4)) / th).astype(np.float32)
            d = np.where(liquid & (tn == AIR), (d + term).astype(np.float32), d)
        wantd[s * 4096:(s + 1) * 4096] = np.where(liquid, d, 0)
    assert np.array_equal(got["dDf"].view(np.uint32), wantd.view(np.uint32))
    # the coarse faces: 4 between uncovered LIQUID coarse cells
    fine_u, coarse_u = _unknowns(sc)
    assert set(np.unique(got["cuc"])) <= {0.0, 4.0}
    assert np.array_equal(got["actc"].astype(bool), coarse_u)


def test_operator_symmetric_positive_and_a1_is_the_dirichlet_diagonal(scene):
    sc = scene
    fine_u, coarse_u = _unknowns(sc)
    rng = np.random.default_rng(7)
    x = [np.where(fine_u, rng.standard_normal(fine_u.size), 0).astype(np.float32),
         np.where(coarse_u, rng.standard_normal(coarse_u.size), 0).astype(np.float32)]
    y = [np.where(fine_u, rng.standard_normal(fine_u.size), 0).astype(np.float32),
         np.where(coarse_u, rng.standard_normal(coarse_u.size), 0).astype(np.float32)]
    Ax, Ay = osp.apply(sc, *x), osp.apply(sc, *y)
    dot = lambda a, b: float(np.dot(a[0].astype(np.float64), b[0]) + np.dot(a[1].astype(np.float64), b[1]))
    assert abs(dot(x, Ay) - dot(y, Ax)) <= 1e-5 * abs(dot(x, Ay))
    assert dot(x, Ax) > 0 and dot(y, Ay) > 0
    one = [fine_u.astype(np.float32), coarse_u.astype(np.float32)]
    q = osp.apply(sc, *one)
    c = osp.coefficients(sc)
    np.testing.assert_allclose(q[0][fine_u], c["dDf"][fine_u], rtol=1e-5, atol=1e-4)
    np.testing.assert_allclose(q[1][coarse_u], c["dDc"][coarse_u], rtol=1e-5, atol=1e-4)


def test_vcycle_scales_exactly(scene):
    sc = scene
    fine_u, coarse_u = _unknowns(sc)
    rng = np.random.default_rng(3)
    rf = np.where(fine_u, rng.standard_normal(fine_u.size), 0).astype(np.float32)
    rc = np.where(coarse_u, rng.standard_normal(coarse_u.size), 0).astype(np.float32)
    z1 = osp.vcycle(sc, rf, rc)
    z2 = osp.vcycle(sc, np.float32(4) * rf, np.float32(4) * rc)
    assert np.array_equal(z2[0], np.float32(4) * z1[0]) and np.array_equal(z2[1], np.float32(4) * z1[1])
    # a preconditioner: positive on the residual it is given
    assert float(np.dot(z1[0].astype(np.float64), rf) + np.dot(z1[1].astype(np.float64), rc)) > 0


@pytest.mark.parametrize("nb,fallback", [((4, 4, 4), False), ((4, 4, 4), True), ((8, 8, 4), False)])
def test_projection_leaves_only_the_residual_divergence(nb, fallback):
    sc = ss.sparse_basin(nb, seed=2102 + nb[2], warm=True)
    vol = osp.volume(sc)
    tol = 5e-4 if fallback else 1e-5
    info = osp.project(sc, vol * 1.002, tol=tol, maxiter=200, sweeps=1, boost=1.5 if fallback else 1.0,
                       fallback=fallback)
    assert info["status"] == 0 and info["iterations"] > 0
    fine_u, coarse_u = _unknowns(sc)
    # the rhs the projected velocity gives, with the same gamma: -h div u + gamma h^2 = b - A P
    before = ss.sparse_basin(nb, seed=2102 + nb[2], warm=True)
    b0 = osp.rhs(before, info["gamma"])
    b1 = osp.rhs(sc, info["gamma"])
    n0 = np.sqrt(np.sum(b0[0][fine_u].astype(np.float64) ** 2) + np.sum(b0[1][coarse_u].astype(np.float64) ** 2))
    n1 = np.sqrt(np.sum(b1[0][fine_u].astype(np.float64) ** 2) + np.sum(b1[1][coarse_u].astype(np.float64) ** 2))
    assert n1 <= 4 * tol * n0 + 1e-6 * n0, (n1 / n0, tol)
    # valid flags: set exactly on faces with no wall and water on a side (spot check counts)
    assert sc.fuf.sum() > 0 and sc.fuc.sum() > 0


def test_coarse_only_basin():
    """No fine blocks at all: the coarse grid alone (the pools are empty)."""
    sc = ss.sparse_basin((4, 4, 4), seed=2103)
    sc.slot[:] = 0
    sc.where = np.zeros((0, 3), np.int32)
    sc.nslots = 0
    for k in ("tf", "phif", "Pf", "uf", "vf", "wf", "fuf", "fvf", "fwf"):
        setattr(sc, k, getattr(sc, k)[:0].copy())
    vol = osp.volume(sc)
    info = osp.project(sc, vol, tol=1e-5, maxiter=100)
    assert info["status"] == 0 and info["iterations"] > 0
