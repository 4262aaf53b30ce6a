"""The level-set passes on the GPU (redistance!, classify!, filltrapped!) against the oracle.

All three are Float32/byte work the kernels do in the reference's arithmetic, so the
comparison is bit for bit: every level-set value and every cell class, after 0-12 Jacobi
sweeps (redistance!'s step! count is band + 3 = 7, initialize!'s 2 band + 4 = 12), on grids
whose rows take the 4-cells-a-thread form and on ragged ones that take the one-cell form;
and the trapped-air fill at 1, 2 and 32 rounds on scenes with sealed pockets, pockets
joined to the top, and lines long enough to span several chunks of the column sweeps.
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


def _noisy_phi(b, seed, spikes=True):
    """The basin's level set made wavy and noisy (frozen cells, far cells, cells beyond
    phimax), as after particles have splatted into it."""
    n1, n2, n3 = b.grid.n
    rng = np.random.default_rng(seed)
    i = np.arange(n1)[None, None, :]
    j = np.arange(n2)[None, :, None]
    phi = b.phi.reshape(n3, n2, n1) + (0.6 * np.sin(0.7 * i) * np.cos(0.5 * j)) * b.grid.dx
    phi = phi + rng.uniform(-0.3, 0.3, phi.shape) * b.grid.dx
    phi = phi.astype(np.float32).reshape(-1)
    if spikes:
        phi[rng.integers(0, phi.size, phi.size // 50)] *= np.float32(7.0)
    return phi


CASES = {
    "box64": lambda: scene.box_basin(64, seed=31),
    "ragged30x14x18": lambda: scene.box_basin((30, 14, 18), seed=32, wall=0.47),
    "wide96x32x40": lambda: scene.box_basin((96, 32, 40), seed=33, height=0.4),
}


@pytest.mark.parametrize("iterations", [0, 1, 2, 7, 12])
@pytest.mark.parametrize("case", list(CASES))
def test_redistance_classify_bitexact(cuda, case, iterations):
    import torch

    import mpp

    b = CASES[case]()
    phi = _noisy_phi(b, 40 + iterations)
    p = mpp.Projector(b.grid)
    d_phi, d_phi0 = _t(phi, cuda), torch.full_like(_t(phi, cuda), float("nan"))
    types = torch.full((b.grid.ncells,), 255, dtype=torch.uint8, device=cuda)
    out = p.redistance(d_phi, d_phi0, iterations, types=types)
    assert out is (d_phi0 if iterations % 2 else d_phi)
    want = oracle.redistance(b.grid, phi, iterations)
    np.testing.assert_array_equal(_np(out).view(np.uint32), want.view(np.uint32))
    np.testing.assert_array_equal(_np(types), oracle.classify(b.grid, want))


def test_classify_alone(cuda):
    import torch

    import mpp

    b = CASES["ragged30x14x18"]()
    phi = _noisy_phi(b, 7, spikes=False)
    p = mpp.Projector(b.grid)
    types = torch.zeros(b.grid.ncells, dtype=torch.uint8, device=cuda)
    p.classify(types, _t(phi, cuda))
    np.testing.assert_array_equal(_np(types), oracle.classify(b.grid, phi))


def _pocketed(shape, seed, air=0.3):
    """A basin whose water holds random air cells (sealed pockets and pockets that join
    the surface), with phi positive on the air as classify! would leave it."""
    b = scene.box_basin(shape, seed=seed, height=0.75, wall=0.48)
    n1, n2, n3 = b.grid.n
    T = b.types.reshape(n3, n2, n1).copy()
    rng = np.random.default_rng(seed)
    T[(T == scene.LIQUID) & (rng.random(T.shape) < air)] = scene.AIR
    # a shaft from the top down, with a gallery off it: reached only through several rounds
    T[n3 // 3:, n2 // 2, n1 // 2] = scene.AIR
    T[n3 // 3, n2 // 2, n1 // 2:n1 - 3] = scene.AIR
    T[n3 // 3:n3 // 2, n2 // 2, n1 - 4] = scene.AIR
    phi = b.phi.reshape(n3, n2, n1).copy()
    phi[T == scene.AIR] = np.abs(phi[T == scene.AIR]) + np.float32(0.01)
    return b.grid, T.reshape(-1), phi.reshape(-1).astype(np.float32)


@pytest.mark.parametrize("maxrounds", [0, 1, 2, 32])
@pytest.mark.parametrize("shape", [(64, 64, 64), (40, 36, 44), (32, 16, 288), (16, 288, 32)])
def test_filltrapped_bitexact(cuda, shape, maxrounds):
    import mpp

    g, T, phi = _pocketed(shape, seed=sum(shape) + maxrounds)
    p = mpp.Projector(g)
    dT, dphi = _t(T, cuda), _t(phi, cuda)
    rounds = p.filltrapped(dT, dphi, maxrounds)
    wt, wphi, wr = oracle.filltrapped(g, T, phi, maxrounds)
    assert rounds == wr
    np.testing.assert_array_equal(_np(dT), wt)
    np.testing.assert_array_equal(_np(dphi).view(np.uint32), wphi.view(np.uint32))
    # twice in a row on one context: the masks and round state start afresh
    dT, dphi = _t(T, cuda), _t(phi, cuda)
    assert p.filltrapped(dT, dphi, maxrounds) == wr
    np.testing.assert_array_equal(_np(dT), wt)


def test_step_sequence_on_a_flip_basin(cuda):
    """step!'s level-set phase (src/flip.jl:1399-1401) through the FlipBasin functions:
    redistance! (band + 3 sweeps, the arrays swapped as the reference's), classify!,
    filltrapped!, each bit for bit."""
    import mpp

    b = scene.box_basin(64, seed=77, height=0.7)
    g = b.grid
    phi = _noisy_phi(b, 77)
    b.phi = phi
    s = mpp.FlipBasin.from_scene(b)
    mpp.redistance(s)
    want = oracle.redistance(g, phi, s.band + 3)
    np.testing.assert_array_equal(_np(s.phi).view(np.uint32), want.view(np.uint32))
    mpp.classify(s)
    wt = oracle.classify(g, want)
    np.testing.assert_array_equal(_np(s.types), wt)
    mpp.filltrapped(s)
    ft, fphi, fr = oracle.filltrapped(g, wt, want, 32)
    assert s.trap_rounds == fr
    np.testing.assert_array_equal(_np(s.types), ft)
    np.testing.assert_array_equal(_np(s.phi).view(np.uint32), fphi.view(np.uint32))
