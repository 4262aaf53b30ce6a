"""Batches of basins in one graph launch (mpp_batch_project) and the autotuner."""
import numpy as np
import pytest

from mpp import scene

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _small_batch():
    sizes = [(16, 0.4, 0.45), (32, 0.6, 0.40), (48, 0.7, 0.36), (16, 0.3, 0.47), (64, 0.5, 0.42), (32, 0.8, 0.35)]
    return [scene.box_basin(n, seed=6000 + i, height=h, wall=w) for i, (n, h, w) in enumerate(sizes)]


@pytest.mark.parametrize("grouped", [True, False])
@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_batch_equals_one_by_one(cuda, precision, grouped):
    """One graph launch for all basins gives each basin's own project! bit for bit, whether
    basins of one size run as a group (one launch a pass for all of them) or as chains."""
    import mpp
    from mpp.batch import Batch

    basins = _small_batch()
    batch = Batch(basins, tol=1e-6, maxiter=100, precision=precision)
    batch.set_grouped(grouped)
    for _ in range(2):  # the second call reuses the captured graph (warm starts from the first)
        res = batch.project(1 / 48)
        ones = []
        assert all(r.status == 0 for r in res), [r.as_dict() for r in res]
    assert batch.groups == (2 if grouped else 0)  # the two 16^3 and the two 32^3 basins
    for i, b in enumerate(basins):
        s = mpp.FlipBasin.from_scene(b, tol=1e-6, maxiter=100, precision=precision, graph=True)
        its = []
        for _ in range(2):
            mpp.project(s, 1 / 48)
            its.append(s.iterations[-1])
        a = batch.arrays[i]
        for k in ("u", "v", "w", "fu", "fv", "fw", "P"):
            np.testing.assert_array_equal(_np(a[k]), _np(getattr(s, k)), err_msg=f"basin {i} {k}")
        assert [it[i] for it in batch.iterations] == its
        ones.append(its)


def test_batch_with_fallback(cuda):
    """Basins with the FGMRES fallback finish on the host after the graph launch."""
    import ctypes

    import mpp
    from mpp import _lib
    from mpp.batch import Batch

    basins = _small_batch()[:3]
    batch = Batch(basins, tol=1e-6, maxiter=100, fallback=True)
    for i in range(len(basins)):  # hold CG to 2 iterations so FGMRES takes over
        o = _lib.Opts()
        batch.lib.mpp_opts_default(ctypes.byref(o))
        o.tol, o.maxiter, o.graph, o.fallback, o.cg_maxiter_with_fallback = 1e-6, 100, 1, 1, 2
        _lib.check(batch.lib.mpp_ctx_set_opts(batch.ctx(i), ctypes.byref(o)))
    res = batch.project(1 / 48)
    for r in res:
        assert r.status == 0 and r.fallback_used == 1 and r.true_rel_residual <= 1e-6, r.as_dict()
    # the divergence of the result is that of the pressure solve
    for i, b in enumerate(basins):
        s = mpp.FlipBasin.from_scene(b, tol=1e-6, maxiter=100)
        mpp.project(s, 1 / 48)
        P1, P2 = _np(batch.arrays[i]["P"]), _np(s.P)
        assert np.linalg.norm(P1 - P2) / np.linalg.norm(P2) <= 5e-3


def test_autotune(cuda):
    from mpp.batch import Batch

    basins = [scene.box_basin(64, seed=6100 + i) for i in range(2)] + [scene.box_basin(32, seed=6102)]
    batch = Batch(basins, tol=1e-6, maxiter=100)
    report = batch.autotune()
    assert set(report) == {(64, 64, 64), (32, 32, 32)}
    for dims, rep in report.items():
        assert rep["chosen"] is not None
        assert len(rep["table"]) >= 20  # the forms, then fine x coarse-level sweeps
        # the batch-level pass timed the fastest few single-basin candidates and kept the
        # fastest of those with the whole batch in flight
        conv = [(r["smoother"], r["coarse_smoother"], r["sweeps"], r["sweeps_coarse"], r["coarse_sweeps"])
                for r in sorted((r for r in rep["table"] if r["status"] == 0), key=lambda r: r["ms"])]
        timed = {tuple(int(x) if x.isdigit() else x for x in k.split(",")): v for k, v in rep["batch_ms"].items()}
        assert set(timed) <= set(conv) and conv[0] in timed
        # the fastest with the batch in flight (the timings are rounded: ties allowed)
        assert timed[rep["chosen"]] == min(timed.values())
    # then the grouping: chains, or groups of 4, 8, 16 basins, the fastest kept
    assert batch.grouping is not None and set(batch.grouping["batch_ms"]) == {"0", "4", "8", "16"}
    assert batch.grouping["chosen"] == batch.max_group
    res = batch.project(1 / 48)
    assert all(r.status == 0 for r in res)


def test_batched_workload(cuda):
    """The batched configuration: 48 basins, edges from {48, 64, 96, 128}, one launch."""
    from mpp.batch import Batch

    basins = scene.batch_basins()
    batch = Batch(basins, tol=1e-6, maxiter=100)
    res = batch.project(1 / 48)
    assert len(res) == 48
    assert all(r.status == 0 and r.true_rel_residual <= 2e-6 for r in res), [r.as_dict() for r in res if r.status]


@pytest.mark.parametrize("forms", [("vector", "vector"), ("column", "column"), ("async", "vector")])
def test_grouped_forms_and_uneven_iterations(cuda, forms):
    """Groups of basins converging after different iteration counts (the done ones skip the
    remaining passes) equal each basin's own solve, for the forms a group may run."""
    import mpp
    from mpp.batch import Batch

    basins = [scene.box_basin(32, seed=6300 + i, height=h, wall=w)
              for i, (h, w) in enumerate([(0.3, 0.45), (0.8, 0.40), (0.55, 0.36), (0.7, 0.47)])]
    batch = Batch(basins, tol=1e-7, maxiter=100, precision="fp16")
    for i in range(len(basins)):
        from mpp import _lib

        _lib.check(batch.lib.mpp_ctx_set_smoothers(batch.ctx(i), *(
            {v: k for k, v in _lib.SMOOTHERS.items()}[f] for f in forms)))
    res = batch.project(1 / 48)
    assert batch.groups == 1
    its = [r.iterations for r in res]
    for i, b in enumerate(basins):
        s = mpp.FlipBasin.from_scene(b, tol=1e-7, maxiter=100, precision="fp16", graph=True)
        s.projector.set_smoothers(*forms)
        mpp.project(s, 1 / 48)
        assert its[i] == s.iterations[-1]
        for k in ("u", "v", "w", "fu", "fv", "fw", "P"):
            np.testing.assert_array_equal(_np(batch.arrays[i][k]), _np(getattr(s, k)), err_msg=f"basin {i} {k}")
