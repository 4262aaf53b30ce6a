"""The level-set passes' oracle (redistance!, classify!, filltrapped!; src/flip.jl:608-760)
pinned.

The reference's tests hold no values for these passes, so the C restatement is checked bit
for bit against a second restatement, pure-Python loops over numpy Float32 scalars written
from the same kernels, on small grids; and for what the passes guarantee: a planar surface's
signed distance is a fixed point of redistancing, closed air under water becomes water, air
joined to the top stays air, and the sweep rounds stop once a round reaches nothing.
"""
import numpy as np
import pytest

import oracle
from mpp import scene

F = np.float32
NB = ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))


def _solid(g, i, j, k):
    px = F(g.lo[0]) + (F(i) + F(0.5)) * F(g.dx)
    py = F(g.lo[1]) + (F(j) + F(0.5)) * F(g.dx)
    pz = F(g.lo[2]) + (F(k) + F(0.5)) * F(g.dx)
    return bool(px * px + py * py > F(g.radius) * F(g.radius) or pz < F(g.floor))


def _jmin(x, y):
    d = F(x - y)
    return x if np.signbit(d) else y


def _jmax(x, y):
    d = F(x - y)
    return y if np.signbit(d) else x


def _eikonal(a, b, c, h):
    a, b = _jmin(a, b), _jmax(a, b)
    b, c = _jmin(b, c), _jmax(b, c)
    a, b = _jmin(a, b), _jmax(a, b)
    d = F(a + h)
    if d > b:
        d = F(F(0.5) * F(F(a + b) + np.sqrt(_jmax(F(F(F(2) * h) * h) - F(F(a - b) * F(a - b)), F(0)))))
        if d > c:
            t = F(F(a + b) + c)
            q = F(F(F(F(a * a) + F(b * b)) + F(c * c)) - F(h * h))
            d = F(F(t + np.sqrt(_jmax(F(F(t * t) - F(F(3) * q)), F(0)))) / F(3))
    return d


def _py_reinit(g, phi, phimax):
    n1, n2, n3 = g.n
    P = phi.reshape(n3, n2, n1)
    out = np.empty_like(P)
    h = F(g.dx)
    inr = lambda a, b, c: 0 <= a < n1 and 0 <= b < n2 and 0 <= c < n3
    for k in range(n3):
        for j in range(n2):
            for i in range(n1):
                c = P[k, j, i]
                if _solid(g, i, j, k):
                    lowest, found = c, False
                    for m in range(6):
                        a, b, cc = i + NB[m][0], j + NB[m][1], k + NB[m][2]
                        if inr(a, b, cc) and not _solid(g, a, b, cc):
                            f = P[cc, b, a]
                            lowest = _jmin(lowest, f) if found else f
                            found = True
                    out[k, j, i] = lowest if found else (phimax if c > phimax else (-phimax if c < -phimax else c))
                else:
                    inside = c < 0
                    frozen = False
                    ax = ay = az = phimax
                    for m in range(6):
                        a, b, cc = i + NB[m][0], j + NB[m][1], k + NB[m][2]
                        if inr(a, b, cc) and not _solid(g, a, b, cc):
                            f = P[cc, b, a]
                            if (f < 0) != inside:
                                frozen = True
                            d = F(abs(f))
                            if m < 2:
                                ax = _jmin(ax, d)
                            elif m < 4:
                                ay = _jmin(ay, d)
                            else:
                                az = _jmin(az, d)
                    if frozen:
                        out[k, j, i] = c
                    else:
                        d = _jmin(_eikonal(ax, ay, az, h), phimax)
                        out[k, j, i] = -d if inside else d
    return out.reshape(-1)


def _py_redistance(g, phi, iterations):
    phimax = F(F(iterations + 1) * F(g.dx))
    phi = phi.astype(F)
    for _ in range(iterations):
        phi = _py_reinit(g, phi, phimax)
    return phi


def _py_filltrapped(g, types, phi, maxrounds):
    n1, n2, n3 = g.n
    T = types.reshape(n3, n2, n1).copy()
    Pf = phi.reshape(n3, n2, n1).copy()
    R = np.zeros_like(T)
    R[n3 - 1] = T[n3 - 1] == scene.AIR
    rounds = 0
    for _ in range(maxrounds):
        changed = 0
        for axis in (2, 0, 1):
            others = [a for a in range(3) if a != axis]
            for b in range(g.n[others[1]]):
                for a in range(g.n[others[0]]):
                    L = g.n[axis]
                    for pas in (0, 1):
                        carry = False
                        for m in range(L):
                            l = m if pas == 0 else L - 1 - m
                            c = [0, 0, 0]
                            c[axis], c[others[0]], c[others[1]] = l, a, b
                            idx = (c[2], c[1], c[0])
                            if T[idx] == scene.AIR:
                                if R[idx]:
                                    carry = True
                                elif carry:
                                    R[idx] = 1
                                    changed += 1
                            else:
                                carry = False
        rounds += 1
        if changed == 0:
            break
    fill = (T == scene.AIR) & (R == 0)
    depth = F(F(2) * F(g.dx))
    T[fill] = scene.LIQUID
    for idx in zip(*np.nonzero(fill)):
        Pf[idx] = _jmin(Pf[idx], -depth)
    return T.reshape(-1), Pf.reshape(-1), rounds


def _grid(n, wall=0.45, floor=0.0, dx=0.05):
    n = (n, n, n) if isinstance(n, int) else n
    return scene.Grid(lo=(float(F(-n[0] * dx / 2)), float(F(-n[1] * dx / 2)), 0.0), dx=float(F(dx)), n=n,
                      radius=float(F(wall * n[0] * dx)), floor=floor, levels=2)


@pytest.mark.parametrize("iterations", [1, 2, 5])
def test_redistance_c_matches_python_loops(iterations):
    g = _grid((10, 9, 8), floor=0.06)
    rng = np.random.default_rng(iterations)
    # a wavy surface plus noise: frozen cells, far cells, clamped cells and solid cells
    x, y, z = np.meshgrid(np.arange(10), np.arange(9), np.arange(8), indexing="xy")
    phi = ((z.transpose(2, 0, 1) - 4.0 + 0.7 * np.sin(x.transpose(2, 0, 1))) * g.dx
           + rng.uniform(-0.02, 0.02, (8, 9, 10))).astype(F).reshape(-1)
    phi[::7] *= F(9)  # some values beyond phimax
    got = oracle.redistance(g, phi, iterations)
    want = _py_redistance(g, phi, iterations)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_classify():
    b = scene.box_basin(12, seed=3)
    t = oracle.classify(b.grid, b.phi)
    np.testing.assert_array_equal(t, b.types)  # the scene generator classifies the same way


def _bubbly(n=12, seed=0):
    """A basin with sealed air pockets under water, a pocket joined to the top by a bent
    channel, and random air noise."""
    b = scene.box_basin(n, seed=seed, height=0.7, wall=0.48)
    g = b.grid
    T = b.types.reshape(n, n, n).copy()
    rng = np.random.default_rng(seed)
    liquid = T == scene.LIQUID
    noise = rng.random(T.shape) < 0.25
    T[liquid & noise] = scene.AIR
    phi = b.phi.reshape(n, n, n).copy()
    phi[T == scene.AIR] = np.abs(phi[T == scene.AIR]) + F(0.01)
    return g, T.reshape(-1), phi.reshape(-1).astype(F)


@pytest.mark.parametrize("maxrounds", [1, 2, 32])
@pytest.mark.parametrize("seed", [0, 1])
def test_filltrapped_c_matches_python_loops(seed, maxrounds):
    g, T, phi = _bubbly(12, seed)
    t_c, p_c, r_c = oracle.filltrapped(g, T, phi, maxrounds)
    t_p, p_p, r_p = _py_filltrapped(g, T, phi, maxrounds)
    assert r_c == r_p
    np.testing.assert_array_equal(t_c, t_p)
    np.testing.assert_array_equal(p_c.view(np.uint32), p_p.view(np.uint32))


def test_planar_surface_is_a_fixed_point():
    """phi = z - h at the cell centres is already a distance: redistancing keeps it on the
    non-solid cells within phimax (solid cells take their lowest wet neighbour)."""
    b = scene.box_basin(16, seed=5, height=0.5)
    it = 7
    out = oracle.redistance(b.grid, b.phi, it)
    phimax = F(F(it + 1) * F(b.grid.dx))
    live = b.types != scene.SOLID
    want = np.clip(b.phi, -phimax, phimax)
    np.testing.assert_allclose(out[live], want[live], rtol=0, atol=2e-6)


def test_sealed_bubble_fills_and_open_pocket_stays():
    n = 16
    b = scene.box_basin(n, seed=9, height=0.75, wall=0.48)
    g = b.grid
    T = b.types.reshape(n, n, n).copy()
    phi = b.phi.reshape(n, n, n).copy()
    T[3:5, 7:9, 7:9] = scene.AIR  # sealed bubble near the floor
    phi[3:5, 7:9, 7:9] = F(0.02)
    T[4:, 4, 4] = scene.AIR  # a shaft from the top down to k = 4, then a pocket off it
    T[4, 4, 5:7] = scene.AIR
    phi[T == scene.AIR] = np.maximum(phi[T == scene.AIR], F(0.01))
    t, p, rounds = oracle.filltrapped(g, T.reshape(-1), phi.reshape(-1), 32)
    t = t.reshape(n, n, n)
    p = p.reshape(n, n, n)
    assert (t[3:5, 7:9, 7:9] == scene.LIQUID).all()
    assert (p[3:5, 7:9, 7:9] <= -2 * F(g.dx)).all()
    assert (t[4:, 4, 4] == scene.AIR).all() and (t[4, 4, 5:7] == scene.AIR).all()
    assert 2 <= rounds < 32


def test_rounds_stop_when_nothing_is_reached():
    g, T, phi = _bubbly(12, 2)
    _, _, r_all = oracle.filltrapped(g, T, phi, 32)
    t1, _, r1 = oracle.filltrapped(g, T, phi, r_all)
    t2, _, _ = oracle.filltrapped(g, T, phi, 32)
    assert r1 == r_all
    np.testing.assert_array_equal(t1, t2)
