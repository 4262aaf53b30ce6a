"""The synthetic basins: geometry, classes, walled faces and the level rule."""
import numpy as np
import pytest

from mpp import scene


@pytest.mark.parametrize("n,levels", [((32, 32, 32), 3), ((48, 48, 48), 4), ((64, 64, 64), 4), ((96, 96, 96), 5),
                                      ((128, 128, 128), 5), ((256, 256, 256), 6), ((384, 384, 256), 7)])
def test_levels_rule(n, levels):
    assert scene.levels_for(n) == levels


def test_uniform_is_counter_based():
    a = scene.uniform(5, 1, 1000)
    b = scene.uniform(5, 1, 2000)
    np.testing.assert_array_equal(a, b[:1000])
    assert a.dtype == np.float32 and a.min() >= -1 and a.max() < 1
    assert not np.array_equal(a, scene.uniform(6, 1, 1000))
    assert abs(a.mean()) < 0.1


def test_box_basin_classes_and_walls():
    b = scene.box_basin(64, seed=1000)
    g = b.grid
    n1, n2, n3 = g.n
    t = b.types.reshape(n3, n2, n1)
    solid = scene.solid_cells(g)
    assert np.array_equal(t == scene.SOLID, solid)
    phi = b.phi.reshape(n3, n2, n1)
    assert np.array_equal(t == scene.LIQUID, ~solid & (phi < 0))
    # the top liquid layer of the 64^3 case is k = 38 (1-based), theta 0.9
    col = t[:, n2 // 2, n1 // 2]
    assert np.flatnonzero(col == scene.LIQUID).max() + 1 == 38
    th = phi[37, 32, 32] / (phi[37, 32, 32] - phi[38, 32, 32])
    assert th == pytest.approx(0.9, abs=1e-4)
    # walled faces are zero: the box edge and every face touching a solid cell
    u = b.u.reshape(n3, n2, n1 + 1)
    assert np.all(u[:, :, 0] == 0) and np.all(u[:, :, -1] == 0)
    walled = solid[:, :, :-1] | solid[:, :, 1:]
    assert np.all(u[:, :, 1:-1][walled] == 0)
    assert np.count_nonzero(u[:, :, 1:-1][~walled]) > 0.99 * np.count_nonzero(~walled)


def test_whirl256_surface_theta():
    """256^3: the top liquid layer is k = 154 (1-based) with theta 0.1: a stiff 1/theta term."""
    g = scene.Grid(lo=(-6.4, -6.4, 0.0), dx=0.05, n=(256, 256, 256), radius=5.76, floor=0.0, levels=6)
    z = scene._centres(g, 2, 256, 0.5)
    phi = z - np.float32(0.6 * 256 * 0.05)
    k = np.flatnonzero(phi < 0).max()
    assert k + 1 == 154
    assert phi[k] / (phi[k] - phi[k + 1]) == pytest.approx(0.1, abs=1e-3)


def test_rankine_profiles():
    r = np.array([1.0, 2.5, 5.0])
    ut = scene.rankine(r, 225.0, 2.5)
    assert ut[2] == pytest.approx(225.0 / (2 * np.pi * 5.0))
    assert ut[0] == pytest.approx(225.0 * 1.0 / (2 * np.pi * 6.25))
    eta = scene.rankine_surface(np.array([2.4999, 2.5001]), 225.0, 2.5)
    assert eta[0] == pytest.approx(eta[1], rel=1e-3)  # continuous at the core edge
