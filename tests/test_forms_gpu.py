"""Every smoother form the autotuner can pick, at the sweep counts it picks, against the oracle.

libmpp has four red-black smoother forms (vector, TMA-staged tiles, per-column, and the
vector form's tiles staged by cp.async, for 16-bit storage), chosen
separately for the fine level and for the coarser row-split levels, and the autotuner also
sets the fine and coarser sweep counts and the coarsest solve's sweeps. The FP32 V-cycle
is compared bit for bit with the oracle's (src/flip.jl:992-1014, per-level sweep counts as
the oracle's ORC_SWEEPS), for every fine x coarse form pair, at the reference's counts and
at the autotuner's; whole FP32 solves within the parity tolerance. The 16-bit forms have no
oracle counterpart bit for bit (they store in 16 bits): their forms must agree with each
other exactly. Then the headline configuration (the 256^3 whirlpool) in FP32 against the
oracle, its autotuned FP16 form against the FP64 form, and each member of an autotuned
batch against the oracle at the settings the autotuner chose for it.
"""
import itertools

import numpy as np
import pytest

import oracle
from mpp import scene

pytestmark = pytest.mark.gpu

FORMS = ["vector", "tma", "column", "async"]
PAIRS = list(itertools.product(FORMS, FORMS))
SWEEPS = [(2, 0, 40), (5, 6, 10), (1, 3, 4)]  # (fine, coarser levels, coarsest); 0 = the fine count
PRESSURE_RTOL = 1e-4


def _t(a, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _np(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def basins():
    # 64^3: TMA tiles on the fine level; 128^3: on the fine level and level 1
    return {n: scene.box_basin(n, seed=2000 + n) for n in (64, 128)}


def _projector(grid, fine, coarse, sweeps, sweeps_coarse, csweeps, **kw):
    import mpp

    p = mpp.Projector(grid, sweeps=sweeps, coarse=csweeps, **kw)
    p.set(sweeps_coarse=sweeps_coarse)
    p.set_smoothers(fine, coarse)
    assert p.smoothers() == (fine, coarse)
    return p


@pytest.mark.parametrize("sw", SWEEPS, ids=lambda s: "sweeps%d-%d-%d" % s)
@pytest.mark.parametrize("fine,coarse", PAIRS)
@pytest.mark.parametrize("n", [64, 128])
def test_vcycle_forms_bitexact(cuda, basins, n, fine, coarse, sw):
    b = basins[n]
    p = _projector(b.grid, fine, coarse, *sw)
    r = scene.uniform(12, 5, b.grid.ncells) * (b.types == scene.LIQUID)
    z = _np(p.vcycle(_t(r, cuda), _t(b.types, cuda), _t(b.phi, cuda)))
    d = oracle.diag(b.grid, b.types, b.phi)
    zo = oracle.vcycle(b.grid, r, b.types, d, sweeps=sw[0], sweeps_coarse=sw[1], coarse=sw[2])
    np.testing.assert_array_equal(z, zo)


@pytest.mark.parametrize("prec", ["fp16", "bf16"])
@pytest.mark.parametrize("sw", SWEEPS[:2], ids=lambda s: "sweeps%d-%d-%d" % s)
def test_vcycle_16bit_forms_agree(cuda, basins, prec, sw):
    """The forms do the same arithmetic per cell in the same order: same values."""
    b = basins[128]
    r = scene.uniform(13, 5, b.grid.ncells) * (b.types == scene.LIQUID)
    rt, tt, pt = _t(r, cuda), _t(b.types, cuda), _t(b.phi, cuda)
    out = {}
    for fine, coarse in PAIRS:
        p = _projector(b.grid, fine, coarse, *sw, precision=prec)
        out[(fine, coarse)] = _np(p.vcycle(rt, tt, pt))
    ref = out[("vector", "vector")]
    assert np.isfinite(ref).all() and np.abs(ref).max() > 0
    for k, z in out.items():
        np.testing.assert_array_equal(z, ref, err_msg=f"forms {k}")


@pytest.mark.parametrize("sw", SWEEPS[:2], ids=lambda s: "sweeps%d-%d-%d" % s)
@pytest.mark.parametrize("fine,coarse", PAIRS)
def test_pressure_forms_match_oracle(cuda, basins, fine, coarse, sw):
    b = basins[64]
    tol = 1e-6
    bvec = oracle.rhs(b.grid, b.u, b.v, b.w, b.types, np.float32(0.0))
    P0 = np.zeros(b.grid.ncells, np.float32)
    Po, info = oracle.pressure(b.grid, P0, bvec, b.types, b.phi, tol=tol, maxiter=100, sweeps=sw[0],
                               sweeps_coarse=sw[1], coarse=sw[2])
    p = _projector(b.grid, fine, coarse, *sw, tol=tol, maxiter=100, graph=True)
    P = _t(P0, cuda)
    res = p.pressure(P, _t(bvec, cuda), _t(b.types, cuda), _t(b.phi, cuda))
    assert res.status == 0, res.as_dict()
    assert abs(res.iterations - info.iterations) <= 1, (res.iterations, info.iterations)
    Pg = _np(P)
    rel = np.linalg.norm(Pg - Po) / np.linalg.norm(Po)
    assert rel <= PRESSURE_RTOL, rel
    assert res.true_rel_residual <= 2 * tol


def test_tma_graph_equals_host_loop(cuda, basins):
    """The TMA-staged smoother in the graph's device loop and in the host loop: same bits."""
    b = basins[128]
    bvec = _t(oracle.rhs(b.grid, b.u, b.v, b.w, b.types, np.float32(0.0)), cuda)
    out = []
    for graph in (False, True):
        p = _projector(b.grid, "tma", "tma", 2, 0, 40, tol=1e-6, maxiter=100, graph=graph, precision="fp16")
        P = _t(np.zeros(b.grid.ncells, np.float32), cuda)
        res = p.pressure(P, bvec, _t(b.types, cuda), _t(b.phi, cuda))
        assert res.status == 0
        out.append((_np(P), res.iterations))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]


@pytest.fixture(scope="module")
def whirl():
    return scene.config_basin("whirl256")


def test_whirl256_fp32_matches_oracle(cuda, whirl):
    """The headline configuration (256^3, Rankine vortex, tol 1e-6) in the reference's
    arithmetic, against the oracle's whole projection. At this size the two FP32 solves part
    by more than rounding: the oracle sums its dot products in 256-wide FP32 trees as the
    reference does, the library in FP64, and the solve's conditioning amplifies that
    difference in alpha and beta into ~4e-4 of the pressure. Both stop on the same test; so
    the check is the same iteration count (+-1), the same flags, and a pressure at least as
    close to the exact (FP64, tol 1e-12) solution as the oracle's."""
    import mpp

    b = whirl
    vol0 = oracle.volume(b.grid, b.phi) * 1.001
    ref = oracle.project(b, volume0=vol0, dt=1 / 48, tol=1e-6, maxiter=200)
    s = mpp.FlipBasin.from_scene(b, tol=1e-6, maxiter=200, graph=True)
    s.volume0 = vol0
    mpp.project(s, 1 / 48)
    assert abs(s.iterations[-1] - ref["info"].iterations) <= 1, (s.iterations, ref["info"].iterations)
    for got, want in zip((s.fu, s.fv, s.fw), (ref["fu"], ref["fv"], ref["fw"])):
        np.testing.assert_array_equal(_np(got), want)
    s64 = mpp.FlipBasin.from_scene(b, tol=1e-12, maxiter=400, precision="fp64", graph=True)
    s64.volume0 = vol0
    mpp.project(s64, 1 / 48)
    P64 = s64.projector.solution_f64()
    nrm = np.linalg.norm(P64)
    err_gpu = np.linalg.norm(_np(s.P).astype(np.float64) - P64) / nrm
    err_ref = np.linalg.norm(ref["P"].astype(np.float64) - P64) / nrm
    assert err_gpu <= max(err_ref, 1e-4), (err_gpu, err_ref)
    rel = np.linalg.norm(_np(s.P) - ref["P"]) / np.linalg.norm(ref["P"])
    assert rel <= err_gpu + err_ref + 1e-6, (rel, err_gpu, err_ref)


# The contract of the mixed form at the headline's settings: it stops on the reference's test
# (recursive relative residual <= tol) like every form, so its error against the exact solve
# is bounded by the conditioning times the tolerance, not by the 16-bit storage. At 256^3 with
# the autotuned sweeps it stops after ~8 iterations with a FP64-form error of about 2e-4 (the
# FP32 form at the reference's sweeps needs ~16 and lands nearer); the bound below is that
# contract's. Tightening tol brings the same form under 1e-4: the storage is not the limit.
HEADLINE_FP64_ERROR_BOUND = 5e-4


def test_whirl256_autotuned_fp16_against_fp64(cuda, whirl):
    import torch

    import mpp

    b = whirl
    g = b.grid
    T = lambda a: _t(a, cuda)
    u0, v0, w0, types, phi = T(b.u), T(b.v), T(b.w), T(b.types), T(b.phi)
    P = torch.zeros(g.ncells, dtype=torch.float32, device=cuda)
    flags = [torch.zeros(a.numel(), dtype=torch.uint8, device=cuda) for a in (u0, v0, w0)]

    def run(proj):
        u, v, w = u0.clone(), v0.clone(), w0.clone()
        P.zero_()
        vol0 = proj.volume(phi)
        res = proj.project(u, v, w, *flags, P, types, phi, vol0, 1 / 48)
        return res, _np(P).astype(np.float64)

    p64 = mpp.Projector(g, tol=1e-12, maxiter=400, precision="fp64", graph=True)
    r64, _ = run(p64)
    assert r64.status == 0
    P64 = p64.solution_f64()
    del p64
    proj = mpp.Projector(g, tol=1e-6, maxiter=200, precision="fp16", graph=True)
    tune = proj.autotune(u0, v0, w0, types, phi)
    assert tune["chosen"] is not None
    res, Pm = run(proj)
    assert res.status == 0, res.as_dict()
    assert res.true_rel_residual <= 1.5e-6, res.as_dict()
    err = np.linalg.norm(Pm - P64) / np.linalg.norm(P64)
    assert err <= HEADLINE_FP64_ERROR_BOUND, (err, tune["chosen"])
    proj.set(tol=1e-7)
    res, Pm = run(proj)
    assert res.status == 0
    err7 = np.linalg.norm(Pm - P64) / np.linalg.norm(P64)
    assert err7 <= 1e-4, (err7, tune["chosen"])


def test_autotuned_batch_members_match_oracle(cuda):
    """Each basin of an autotuned batch (its forms and sweeps as the autotuner left them)
    against the oracle's projection at those sweeps."""
    from mpp.batch import Batch

    sizes = [(48, 0.5, 0.40), (64, 0.7, 0.44), (96, 0.4, 0.37), (48, 0.3, 0.47), (64, 0.6, 0.36)]
    basins = [scene.box_basin(n, seed=7000 + i, height=h, wall=w) for i, (n, h, w) in enumerate(sizes)]
    batch = Batch(basins, tol=1e-6, maxiter=100, precision="fp32")
    report = batch.autotune(refine=3)
    res = batch.project(1 / 48)
    for i, b in enumerate(basins):
        chosen = report[tuple(b.grid.n)]["chosen"]
        assert chosen is not None
        fine, coarse, sw, swc, csw = chosen
        ref = oracle.project(b, volume0=batch.volume0[i], dt=1 / 48, tol=1e-6, maxiter=100, sweeps=sw,
                             sweeps_coarse=swc, coarse=csw)
        assert res[i].status == 0
        assert abs(res[i].iterations - ref["info"].iterations) <= 1, (i, chosen, res[i].iterations,
                                                                      ref["info"].iterations)
        a = batch.arrays[i]
        P = _np(a["P"])
        rel = np.linalg.norm(P - ref["P"]) / np.linalg.norm(ref["P"])
        assert rel <= PRESSURE_RTOL, (i, chosen, rel)
        for k in ("fu", "fv", "fw"):
            np.testing.assert_array_equal(_np(a[k]), ref[k])
