"""Host logic of batches: the workload generator, LPT partition, and the multi-rank split
with world_size 2 over gloo (basins are independent: ranks exchange only the results)."""
import os

import numpy as np
import pytest

from mpp import scene
from mpp.batch import basin_cost, lpt_partition


def test_batch_workload_is_deterministic():
    a = scene.batch_basins(8, seed=7)
    b = scene.batch_basins(8, seed=7)
    for x, y in zip(a, b):
        assert x.grid.n == y.grid.n
        np.testing.assert_array_equal(x.u, y.u)
        np.testing.assert_array_equal(x.types, y.types)
    full = scene.batch_basins()
    assert len(full) == 48
    assert {bb.grid.n[0] for bb in full} <= set(scene.BATCH_EDGES)
    for bb in full:
        assert bb.grid.levels == scene.levels_for(bb.grid.n)
        lf = bb.liquid_fraction
        assert 0.05 < lf < 0.8


@pytest.mark.parametrize("nranks", [1, 2, 3, 8])
def test_lpt_partition(nranks):
    rng = np.random.default_rng(nranks)
    costs = rng.uniform(1, 10, 48)
    parts = lpt_partition(costs, nranks)
    assert sorted(i for p in parts for i in p) == list(range(48))
    loads = [costs[p].sum() for p in parts]
    # LPT's bound: the largest load is within 4/3 of the optimum, which is >= the mean
    assert max(loads) <= 4 / 3 * max(costs.sum() / nranks, costs.max()) + 1e-9


def _small_batch():
    sizes = [(16, 0.5, 0.45), (32, 0.6, 0.40), (24, 0.7, 0.36), (16, 0.3, 0.47), (32, 0.5, 0.42), (24, 0.8, 0.35),
             (16, 0.65, 0.41)]
    return [scene.box_basin(n, seed=800 + i, height=h, wall=w) for i, (n, h, w) in enumerate(sizes)]


def oracle_solve(basins, indices, *, dt, tol, maxiter):
    """A rank's share solved on the CPU by the oracle's projection (the test's stand-in for
    the rank's GPU; the partition and the gathering are the product's)."""
    import oracle

    out = []
    for i in indices:
        r = oracle.project(basins[i], dt=dt, tol=tol, maxiter=maxiter)
        info = r["info"]
        out.append(dict(iterations=int(info.iterations), status=0 if info.converged else 1,
                        true_rel_residual=float(info.rnorm / info.bnorm) if info.bnorm else 0.0, fallback_used=0))
    return out


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    from mpp.batch import project_partitioned

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    basins = _small_batch()
    res = project_partitioned(basins, rank, world, solve=oracle_solve, dt=1 / 48, tol=1e-6, maxiter=100)
    # max over ranks of a per-rank time, as the benchmark reports it
    import torch

    t = torch.tensor([float(rank + 1)])
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put(([(o.index, o.rank, o.iterations, o.status) for o in res], float(t)))
    dist.destroy_process_group()


def test_two_ranks_split_a_batch():
    """Two gloo ranks each project their LPT share (the oracle standing in for a rank's GPU)
    and gather the per-basin results: every basin solved once, by the rank the partition
    gave it, with the iterations a serial solve of the whole batch gives."""
    import multiprocessing as mp
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, tmax = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    basins = _small_batch()
    parts = lpt_partition([basin_cost(b) for b in basins], 2)
    assert all(parts)  # both ranks have work
    serial = oracle_solve(basins, range(len(basins)), dt=1 / 48, tol=1e-6, maxiter=100)
    assert [g[0] for g in got] == list(range(len(basins)))
    for i, r_, its, st in got:
        assert i in parts[r_]
        assert its == serial[i]["iterations"] and st == 0
    assert tmax == 2.0


def test_partitioned_single_rank_and_errors():
    from mpp.batch import project_partitioned

    basins = _small_batch()[:3]
    res = project_partitioned(basins, 0, 1, solve=oracle_solve, dt=1 / 48, tol=1e-6, maxiter=100)
    assert [o.index for o in res] == [0, 1, 2] and all(o.rank == 0 for o in res)
    # a rank that drops a basin of its share is an error, not a silent gap
    with pytest.raises(RuntimeError, match="solved 2 of its 3"):
        project_partitioned(basins, 0, 1, solve=lambda b, idx, **kw: oracle_solve(b, idx[:-1], **kw), dt=1 / 48,
                            tol=1e-6, maxiter=100)
    # results gathered twice for one basin are refused
    with pytest.raises(RuntimeError, match="solved twice"):
        project_partitioned(basins, 0, 2, solve=oracle_solve, gather=lambda p: [p, p], dt=1 / 48, tol=1e-6,
                            maxiter=100)
