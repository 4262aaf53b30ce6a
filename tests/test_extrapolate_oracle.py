"""The oracle's extrapolate! (src/flip.jl:1158-1206) against a second, pure-Python
restatement of the same kernels at small sizes (bit for bit, Float32 arithmetic through
numpy scalars), and against what the reference's pass structure implies at a larger size:
the reached set grows by one face-graph layer a pass, unreached and walled faces are zero,
and flagged faces keep their values."""
import numpy as np
import pytest

import oracle
from mpp import scene

F = np.float32


def _issolidcell(g, i, j, k):
    # cellcentre / issolid (src/flip.jl:64-66), Float32; 0-based i is the reference's i - 1
    px = F(g.lo[0]) + F(F(i) + F(0.5)) * F(g.dx)
    py = F(g.lo[1]) + F(F(j) + F(0.5)) * F(g.dx)
    pz = F(g.lo[2]) + F(F(k) + F(0.5)) * F(g.dx)
    return F(px * px) + F(py * py) > F(F(g.radius) * F(g.radius)) or pz < F(g.floor)


def _walled(g, f, axis):
    # walled (src/flip.jl:784-789)
    if f[axis] == 0 or f[axis] == g.n[axis]:
        return True
    b = list(f)
    b[axis] -= 1
    return _issolidcell(g, *b) or _issolidcell(g, *f)


NB = ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))


def _py_extrapolate(g, arrs, flags, layers):
    """extrapolate_kernel!, unreached_kernel! and solidify! as loops (src/flip.jl:1161-1206)."""
    arrs = [np.array(a, dtype=F).reshape(g.face_shape(ax)[::-1]).copy() for ax, a in enumerate(arrs)]
    flags = [np.array(a, dtype=np.uint8).reshape(g.face_shape(ax)[::-1]).copy() for ax, a in enumerate(flags)]
    for ax in range(3):
        a1, a2, a3 = g.face_shape(ax)
        src, fin = arrs[ax], flags[ax]
        for _ in range(layers):
            out, fout = np.empty_like(src), np.empty_like(fin)
            for k in range(a3):
                for j in range(a2):
                    for i in range(a1):
                        if fin[k, j, i]:
                            out[k, j, i], fout[k, j, i] = src[k, j, i], 1
                            continue
                        s, m = F(0), 0
                        if not _walled(g, (i, j, k), ax):
                            for di, dj, dk in NB:
                                x, y, z = i + di, j + dj, k + dk
                                if 0 <= x < a1 and 0 <= y < a2 and 0 <= z < a3 and fin[z, y, x]:
                                    s = F(s + src[z, y, x])
                                    m += 1
                        out[k, j, i] = F(s / F(m)) if m > 0 else src[k, j, i]
                        fout[k, j, i] = 1 if m > 0 else 0
            src, fin = out, fout
        src = np.where(fin == 0, F(0), src)
        arrs[ax], flags[ax] = src, fin
    for ax in range(3):
        a1, a2, a3 = g.face_shape(ax)
        for k in range(a3):
            for j in range(a2):
                for i in range(a1):
                    if _walled(g, (i, j, k), ax):
                        arrs[ax][k, j, i] = F(0)
    return [a.ravel() for a in arrs] + [f.ravel() for f in flags]


def _inputs(g, seed, density):
    rng = np.random.default_rng(seed)
    vel = [rng.uniform(-1, 1, int(np.prod(g.face_shape(a)))).astype(F) for a in range(3)]
    fl = [(rng.random(int(np.prod(g.face_shape(a)))) < density).astype(np.uint8) for a in range(3)]
    return vel, fl


@pytest.mark.parametrize("layers", [0, 1, 2, 3, 6])
@pytest.mark.parametrize("density", [0.02, 0.3])
def test_oracle_matches_loop_restatement(layers, density):
    b = scene.box_basin((10, 8, 6), seed=5000)
    g = b.grid
    vel, fl = _inputs(g, 5 + layers, density)
    got = oracle.extrapolate(g, *vel, *fl, layers=layers)
    want = _py_extrapolate(g, vel, fl, layers)
    for x, y in zip(got, want):
        assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))


def _reach(g, flags, layers):
    """Faces within `layers` steps of a flagged face, stepping only into faces that are not
    walled (a walled face never takes a value, so it never passes one on)."""
    out = []
    for ax in range(3):
        shape = g.face_shape(ax)[::-1]
        r = flags[ax].reshape(shape).astype(bool)
        k, j, i = np.meshgrid(*(np.arange(s) for s in shape), indexing="ij")
        walled = np.vectorize(lambda a, b_, c: _walled(g, (a, b_, c), ax))(i, j, k)
        for _ in range(layers):
            nb = np.zeros_like(r)
            nb[:, :, 1:] |= r[:, :, :-1]
            nb[:, :, :-1] |= r[:, :, 1:]
            nb[:, 1:, :] |= r[:, :-1, :]
            nb[:, :-1, :] |= r[:, 1:, :]
            nb[1:, :, :] |= r[:-1, :, :]
            nb[:-1, :, :] |= r[1:, :, :]
            r = r | (nb & ~walled)
        out.append((r.ravel(), walled.ravel()))
    return out


def test_projection_flags_reach_and_zero():
    """From the projection's own flags at 20^3: the reached set is exactly the faces within
    6 layers; unreached and walled faces are zero; flagged faces keep their values."""
    b = scene.box_basin(20, seed=5001)
    g = b.grid
    pr = oracle.project(b, tol=1e-5, maxiter=200)
    vel = [pr["u"], pr["v"], pr["w"]]
    fl = [pr["fu"], pr["fv"], pr["fw"]]
    got = oracle.extrapolate(g, *vel, *fl, layers=6)
    for ax, (reach, walled) in enumerate(_reach(g, fl, 6)):
        a, f = got[ax], got[3 + ax]
        assert np.array_equal(f.astype(bool), reach)
        assert np.all(a[~reach] == 0) and np.all(a[walled] == 0)
        keep = (fl[ax] != 0) & ~walled
        assert np.array_equal(a[keep], vel[ax][keep])
        assert np.count_nonzero(f) > np.count_nonzero(fl[ax])  # it did carry the water's velocity out


def test_no_layer_keeps_flag_values_and_zeroes():
    """layers = 0: no extrapolate_kernel! runs, so the flags stay byte for byte (any nonzero
    value counts as flagged) and only unreached_kernel! and solidify! act."""
    b = scene.box_basin((10, 8, 6), seed=5002)
    g = b.grid
    rng = np.random.default_rng(11)
    vel = [rng.uniform(-1, 1, int(np.prod(g.face_shape(a)))).astype(F) for a in range(3)]
    fl = [rng.integers(0, 4, int(np.prod(g.face_shape(a)))).astype(np.uint8) for a in range(3)]
    got = oracle.extrapolate(g, *vel, *fl, layers=0)
    for ax in range(3):
        assert np.array_equal(got[3 + ax], fl[ax])
        walled = np.array([_walled(g, (i, j, k), ax) for k in range(g.face_shape(ax)[2])
                           for j in range(g.face_shape(ax)[1]) for i in range(g.face_shape(ax)[0])])
        keep = (fl[ax] != 0) & ~walled
        assert np.array_equal(got[ax][keep], vel[ax][keep])
        assert np.all(got[ax][~keep] == 0)


def test_flagged_walled_face_is_a_source_then_zero():
    """A walled face flagged on entry lends its value to its neighbours in the first layer
    (extrapolate_kernel! reads any flagged neighbour), and solidify! zeroes it at the end."""
    b = scene.box_basin((10, 8, 6), seed=5003)
    g = b.grid
    a1, a2, a3 = g.face_shape(0)
    vel = [np.zeros(int(np.prod(g.face_shape(a))), dtype=F) for a in range(3)]
    fl = [np.zeros(int(np.prod(g.face_shape(a))), dtype=np.uint8) for a in range(3)]
    # a walled u face whose +x neighbour in the same row is not walled (the cylinder's wall)
    j, k = a2 // 2, a3 // 2
    i = next(i for i in range(a1 - 1) if _walled(g, (i, j, k), 0) and not _walled(g, (i + 1, j, k), 0))
    src = i + a1 * (j + a2 * k)
    dst = src + 1
    vel[0][src] = F(0.75)
    fl[0][src] = 1
    got = oracle.extrapolate(g, *vel, *fl, layers=1)
    assert got[0][dst] == F(0.75) and got[3][dst] == 1
    assert got[0][src] == 0 and got[3][src] == 1
