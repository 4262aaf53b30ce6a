"""The sparse basin's CUDA path against the oracle (oracle/sparse.c), through the C ABI.

Bit for bit: the level-0 coefficients and Dirichlet diagonals, the operator, one damped
Jacobi sweep, the right-hand side, the whole V-cycle (coefficients, hierarchy, smoothing,
transfers, coarsest solve) and the gradient update with its flags and face restriction.
Whole solves differ only in the dot products' summation order (FP64 on the GPU, FP32
trees in the oracle): pressure within 1e-4 relative L2, iterations within 1.
"""
import numpy as np
import pytest

from mpp import sparse as msp
from mpp import sparse_scene as ss
from oracle import sparse as osp

pytestmark = pytest.mark.gpu

SCENES = {"4x4x4": dict(nb=(4, 4, 4), seed=2201), "8x8x4": dict(nb=(8, 8, 4), seed=2202),
          "8x8x8_rings": dict(nb=(8, 8, 8), seed=2203, rings=1)}


def _scene(name, warm=True):
    kw = dict(SCENES[name])
    return ss.sparse_basin(kw.pop("nb"), warm=warm, **kw)


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _host(t):
    return t.cpu().numpy()


def _bits_equal(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def _unknowns(sc):
    fine = (sc.tf == 1) & np.repeat(sc.where[:, 0] >= 0, 4096)
    cov = np.zeros(sc.grid.nc, bool)
    for w in sc.where:
        if w[0] >= 0:
            cov[w[0] * 4:w[0] * 4 + 4, w[1] * 4:w[1] * 4 + 4, w[2] * 4:w[2] * 4 + 4] = True
    return fine, (sc.tc == 1) & ~cov.reshape(-1, order="F")


def _used(sc, arr, per):
    """The values of slots in use (free slots hold whatever a kernel never wrote)."""
    m = np.repeat(sc.where[:, 0] >= 0, per)
    return np.asarray(arr)[: m.size][m]


@pytest.mark.parametrize("name", list(SCENES))
def test_coefficients_bitexact(cuda, name):
    sc = _scene(name)
    want = osp.coefficients(sc)
    s = msp.SparseBasin.from_scene(sc)
    s.operator()
    for key, gkey, per in (("cuf", "cu_f", 4352), ("cvf", "cv_f", 4352), ("cwf", "cw_f", 4352), ("dDf", "dD_f", 4096)):
        assert _bits_equal(_used(sc, s.read(gkey), per), _used(sc, want[key], per)), key
    for key, gkey in (("cuc", "cu_c"), ("cvc", "cv_c"), ("cwc", "cw_c"), ("dDc", "dD_c")):
        assert _bits_equal(s.read(gkey), want[key]), key
    # the coarse activity after hierarchy! (uncovered LIQUID cells keep coefficients!'s value)
    fine_u, coarse_u = _unknowns(sc)
    act = s.read("act_c").astype(bool)
    assert np.array_equal(act[coarse_u], want["actc"].astype(bool)[coarse_u])


@pytest.mark.parametrize("name", list(SCENES))
def test_apply_jacobi_rhs_bitexact(cuda, name):
    sc = _scene(name)
    fine_u, coarse_u = _unknowns(sc)
    rng = np.random.default_rng(11)
    xf = np.where(sc.tf != 0, rng.standard_normal(fine_u.size), 0).astype(np.float32)
    xc = np.where(sc.tc != 0, rng.standard_normal(coarse_u.size), 0).astype(np.float32)
    bf = rng.standard_normal(fine_u.size).astype(np.float32)
    bc = rng.standard_normal(coarse_u.size).astype(np.float32)
    s = msp.SparseBasin.from_scene(sc)
    s.operator()
    import torch

    qf, qc = torch.zeros(fine_u.size, device="cuda"), torch.zeros(coarse_u.size, device="cuda")
    s.apply(_dev(xf), _dev(xc), qf, qc)
    wq = osp.apply(sc, xf, xc)
    assert _bits_equal(_used(sc, _host(qf), 4096), _used(sc, wq[0], 4096))
    assert _bits_equal(_host(qc), wq[1])
    # right-hand side (finerhs_kernel! + coarserhs_kernel!)
    gf, gc = torch.zeros(fine_u.size, device="cuda"), torch.zeros(coarse_u.size, device="cuda")
    s.rhs(0.0123, gf, gc)
    wb = osp.rhs(sc, np.float32(0.0123))
    assert _bits_equal(_used(sc, _host(gf), 4096), _used(sc, wb[0], 4096))
    assert _bits_equal(_host(gc), wb[1])


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("sweeps,boost", [(1, 1.0), (2, 1.0), (1, 1.5)])
def test_vcycle_bitexact(cuda, name, sweeps, boost):
    sc = _scene(name)
    fine_u, coarse_u = _unknowns(sc)
    rng = np.random.default_rng(5 + sweeps)
    rf = np.where(fine_u, rng.standard_normal(fine_u.size), 0).astype(np.float32)
    rc = np.where(coarse_u, rng.standard_normal(coarse_u.size), 0).astype(np.float32)
    want = osp.vcycle(sc, rf, rc, sweeps=sweeps, boost=boost)
    s = msp.SparseBasin.from_scene(sc)
    s.operator()
    import torch

    zf, zc = torch.zeros(fine_u.size, device="cuda"), torch.zeros(coarse_u.size, device="cuda")
    s.vcycle(_dev(rf), _dev(rc), zf, zc, sweeps=sweeps, coarse=40, boost=boost)
    assert _bits_equal(_used(sc, _host(zf), 4096), _used(sc, want[0], 4096))
    assert _bits_equal(_host(zc), want[1])


@pytest.mark.parametrize("name", list(SCENES))
def test_gradient_bitexact(cuda, name):
    """The velocity update, valid flags and face restriction from a given pressure."""
    sc = _scene(name)
    fine_u, coarse_u = _unknowns(sc)
    rng = np.random.default_rng(13)
    sc.Pf[:] = np.where(fine_u, rng.standard_normal(fine_u.size), 0).astype(np.float32)
    sc.Pc[:] = np.where(coarse_u, rng.standard_normal(coarse_u.size), 0).astype(np.float32)
    s = msp.SparseBasin.from_scene(sc)
    want = sc.copy()
    osp.gradient(want)
    s.gradient()
    for k, per in (("uf", 4352), ("vf", 4352), ("wf", 4352), ("fuf", 4352), ("fvf", 4352), ("fwf", 4352)):
        assert _bits_equal(_used(sc, _host(getattr(s, k)), per), _used(sc, getattr(want, k), per)), k
    for k in ("uc", "vc", "wc", "fuc", "fvc", "fwc"):
        assert _bits_equal(_host(getattr(s, k)), getattr(want, k)), k


def _rel(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / max(np.linalg.norm(b.astype(np.float64)), 1e-30))


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("graph", [False, True])
def test_project_matches_oracle(cuda, name, graph):
    sc = _scene(name)
    vol = osp.volume(sc)
    want = sc.copy()
    info = osp.project(want, vol * 1.002, tol=1e-5, maxiter=200)
    s = msp.SparseBasin.from_scene(sc, graph=graph, tol=1e-5, maxiter=200)
    assert s.volume0 == pytest.approx(vol, rel=1e-6)
    s.volume0 = vol * 1.002
    msp.project(s, 1 / 48)
    assert s.last.status == 0
    assert abs(s.iterations[-1] - info["iterations"]) <= 1, (s.iterations, info)
    fine_u, coarse_u = _unknowns(sc)
    P = np.concatenate([_host(s.Pf)[fine_u], _host(s.Pc)[coarse_u]])
    W = np.concatenate([want.Pf[fine_u], want.Pc[coarse_u]])
    assert _rel(P, W) <= 1e-4
    for k, per in (("fuf", 4352), ("fvf", 4352), ("fwf", 4352)):
        assert np.array_equal(_used(sc, _host(getattr(s, k)), per), _used(sc, getattr(want, k), per)), k
    for k in ("fuc", "fvc", "fwc"):
        assert np.array_equal(_host(getattr(s, k)), getattr(want, k)), k
    assert s.last.gamma == pytest.approx(info["gamma"], rel=1e-5, abs=1e-9)


def test_graph_equals_host_loop(cuda):
    sc = _scene("8x8x4")
    a = msp.SparseBasin.from_scene(sc, graph=False, tol=1e-6)
    b = msp.SparseBasin.from_scene(sc, graph=True, tol=1e-6)
    msp.project(a, 1 / 48)
    msp.project(b, 1 / 48)
    assert a.iterations == b.iterations
    assert _bits_equal(_host(a.Pf), _host(b.Pf)) and _bits_equal(_host(a.Pc), _host(b.Pc))
    # and the cached graph a second time (warm start from the first solve's P)
    msp.project(b, 1 / 48)
    msp.project(a, 1 / 48)
    assert a.iterations == b.iterations and _bits_equal(_host(a.Pf), _host(b.Pf))


@pytest.mark.parametrize("name", ["4x4x4", "8x8x4"])
def test_fallback_dispatch(cuda, name):
    """The dispatch of src/fgmres.jl:96-110: CG with boost 1.5 and tol 5e-4, FGMRES if the
    true residual misses; either way the true residual meets tol."""
    sc = _scene(name)
    vol = osp.volume(sc)
    want = sc.copy()
    info = osp.project(want, vol, tol=5e-4, maxiter=240, boost=1.5, fallback=True)
    s = msp.SparseBasin.from_scene(sc, fallback=True)
    msp.project(s, 1 / 48)
    assert s.last.status == 0 and s.last.rel_residual <= 5e-4
    assert abs(s.iterations[-1] - info["iterations"]) <= 1
    # a CG capped below what it needs, then FGMRES finishes
    s2 = msp.SparseBasin.from_scene(sc, fallback=True, tol=1e-5, cg_maxiter=1)
    msp.project(s2, 1 / 48)
    assert s2.last.status == 0 and s2.last.rel_residual <= 1e-5 and s2.last.fgmres_iterations > 0


@pytest.mark.parametrize("cap", [0, 2])
def test_fgmres_runs_after_a_capped_cg(cuda, cap):
    sc = _scene("4x4x4")
    fine_u, coarse_u = _unknowns(sc)
    b = osp.rhs(sc, np.float32(0.0))
    want = sc.copy()
    info = osp.pressure(want, b[0], b[1], tol=1e-5, maxiter=240, boost=1.5, fallback=True, cg_maxiter=cap)
    s = msp.SparseBasin.from_scene(sc)
    its = msp.pressure(s, _dev(b[0]), _dev(b[1]), fallback=True, tol=1e-5, maxiter=240, cg_maxiter=cap)
    assert s.last.status == 0 and s.last.rel_residual <= 1e-5
    assert s.last.fgmres_iterations > 0 and info["fgmres_iterations"] > 0
    assert its == s.last.iterations and info["status"] == 0
    assert abs(its - info["iterations"]) <= 2
    P = np.concatenate([_host(s.Pf)[fine_u], _host(s.Pc)[coarse_u]])
    W = np.concatenate([want.Pf[fine_u], want.Pc[coarse_u]])
    assert _rel(P, W) <= 1e-4


def test_coarse_only_basin(cuda):
    sc = ss.sparse_basin((4, 4, 4), seed=2204)
    sc.slot[:] = 0
    sc.where = np.zeros((0, 3), np.int32)
    sc.nslots = 0
    for k in ("tf", "phif", "Pf", "uf", "vf", "wf", "fuf", "fvf", "fwf"):
        setattr(sc, k, getattr(sc, k)[:0].copy())
    vol = osp.volume(sc)
    want = sc.copy()
    info = osp.project(want, vol, tol=1e-5, maxiter=100)
    # an empty pool still needs tensors with a valid address
    import torch

    s = msp.SparseBasin.from_scene(sc, tol=1e-5, maxiter=100)
    for k in ("tf", "phif", "Pf", "uf", "vf", "wf", "fuf", "fvf", "fwf"):
        setattr(s, k, torch.zeros(1, dtype=getattr(s, k).dtype, device="cuda"))
    s.volume0 = vol
    msp.project(s, 1 / 48)
    assert s.last.status == 0 and abs(s.iterations[-1] - info["iterations"]) <= 1
    assert _rel(_host(s.Pc), want.Pc) <= 1e-4
    assert np.array_equal(_host(s.fuc), want.fuc)


def test_not_converged_warns_and_errors(cuda):
    sc = _scene("4x4x4")
    s = msp.SparseBasin.from_scene(sc, tol=1e-9, maxiter=2)
    with pytest.warns(RuntimeWarning, match="did not converge"):
        msp.project(s, 1 / 48)
    assert s.iterations[-1] == 2
    with pytest.raises(msp._lib.MppError):
        msp.project(s, 1 / 48, sweeps=0)
    import ctypes

    a = s.arrays()
    a.nslots = s.capacity + 1
    o = s.options()
    r = msp.SparseResult()
    assert s._lib.mpp_sparse_project(s._ctx, ctypes.byref(a), 1.0, 0.02, 0.5, ctypes.byref(o), ctypes.byref(r),
                                     None) == msp._lib.ERR_INVALID
