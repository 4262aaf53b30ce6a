"""Seeded synthetic sparse basins: the arrays a SparseBasin hands to ``project!``.

The reference's sparse basin (src/sflip.jl) keeps fine 16^3 blocks of cells ``dx`` wide
where the water's surface is, over a dense coarse grid of cells ``4 dx`` wide. Its block
table and pools come from its own refinement and particle code; no dataset exists for the
path. This module makes the same arrays for a cylindrical basin with a whirlpool funnel:

* ``SparseGrid`` geometry (src/sflip.jl:38-66): ``nb`` blocks a side, coarse cells
  ``4 dx`` wide, cell centres at ``lo + (I + 1/2) h``; a cell is SOLID when its centre lies
  outside the cylinder or under the floor, one coarse cell above the grid's bottom;
* the level set ``phi = z - h(r)`` of a funnel-shaped surface, at fine and coarse centres;
* the fine blocks: those holding a coarse cell within 1.5 coarse cells of the surface or
  whose level set changes sign to a neighbour (as ``marksurface_kernel!``,
  src/sflip.jl:385-408), grown by ``rings`` blocks; slots are handed out in block order
  with every ``free_every``-th slot left free (its ``where`` is -1s), as a refinement that
  released blocks leaves the pool;
* classes as ``classifyfine_kernel!``/``classifycoarse_kernel!`` (src/sflip.jl:921-940),
  the coarse level set under fine blocks as their means (``restrictcells_kernel!``,
  src/sflip.jl:584-594);
* face velocities: a swirl about the axis plus uniform noise from the counter-based
  generator of ``scene.uniform``; a warm-start pressure on the water cells if asked.

All arithmetic that decides a cell's class is Float32, as in the reference.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .scene import AIR, LIQUID, SOLID, uniform

BLOCK, RATIO = 16, 4
BCELLS, BFACES = BLOCK ** 3, (BLOCK + 1) * BLOCK * BLOCK


@dataclasses.dataclass
class SparseGrid:
    lo: tuple
    dx: float
    nb: tuple
    radius: float
    floor_z: float

    @property
    def nc(self):
        return tuple(int(b) * RATIO for b in self.nb)


@dataclasses.dataclass
class SparseScene:
    grid: SparseGrid
    slot: np.ndarray    # int32 [nblocks]: 1-based slot of each block, 0 for none
    where: np.ndarray   # int32 [nslots, 3]: each slot's block, -1s for a free slot
    nslots: int
    tf: np.ndarray      # uint8 [nslots*4096]
    tc: np.ndarray      # uint8 coarse (column-major)
    phif: np.ndarray
    phic: np.ndarray
    Pf: np.ndarray
    Pc: np.ndarray
    uf: np.ndarray      # float32 [nslots*BFACES]
    vf: np.ndarray
    wf: np.ndarray
    uc: np.ndarray      # float32 coarse faces, one longer along their axis
    vc: np.ndarray
    wc: np.ndarray
    fuf: np.ndarray
    fvf: np.ndarray
    fwf: np.ndarray
    fuc: np.ndarray
    fvc: np.ndarray
    fwc: np.ndarray
    seed: int = 0

    def copy(self) -> "SparseScene":
        kw = {f.name: getattr(self, f.name) for f in dataclasses.fields(self)}
        for k, v in kw.items():
            if isinstance(v, np.ndarray):
                kw[k] = v.copy()
        return SparseScene(**kw)

    def coarse_shape(self, axis=0):
        n = list(self.grid.nc)
        if axis:
            n[axis - 1] += 1
        return tuple(n)

    @property
    def used_slots(self) -> int:
        return int((self.where[:, 0] >= 0).sum())


def _centres(lo, h, n):
    return (np.float32(lo) + (np.arange(n, dtype=np.float32) + np.float32(0.5)) * np.float32(h)).astype(np.float32)


def _solid(grid: SparseGrid, px, py, pz):
    r2 = np.float32(grid.radius) * np.float32(grid.radius)
    return (px * px + py * py > r2) | (pz < np.float32(grid.floor_z))


def _face_view(pool, s, axis):
    """Slot s's faces along `axis` as a [k, j, i] array (17 along the axis)."""
    f = pool[s * BFACES:(s + 1) * BFACES]
    if axis == 1:
        return f.reshape(BLOCK, BLOCK, BLOCK + 1)
    if axis == 2:
        return f.reshape(BLOCK, BLOCK + 1, BLOCK)
    return f.reshape(BLOCK + 1, BLOCK, BLOCK)


def sync_planes(slot, where, nb, axis, pool):
    """A block's high-plane faces take the low-plane faces of the fine block above it
    (``syncplanes_kernel!``, src/sflip.jl:621-644), so the two copies of a face on a plane
    between fine blocks agree."""
    for s, w in enumerate(where):
        if w[0] < 0:
            continue
        n = [int(v) for v in w]
        n[axis - 1] += 1
        if n[axis - 1] >= nb[axis - 1]:
            continue
        s2 = int(slot[n[0] + nb[0] * (n[1] + nb[1] * n[2])])
        if s2 == 0:
            continue
        hi, lo = _face_view(pool, s, axis), _face_view(pool, s2 - 1, axis)
        if axis == 1:
            hi[:, :, BLOCK] = lo[:, :, 0]
        elif axis == 2:
            hi[:, BLOCK, :] = lo[:, 0, :]
        else:
            hi[BLOCK, :, :] = lo[0, :, :]


def restrict_faces(where, axis, pool, coarse):
    """Coarse faces along `axis` that fine blocks hold: the mean of their 16 fine faces, in
    Float32 as ``restrictfaces_kernel!`` sums them (src/sflip.jl:597-611). ``coarse`` is
    indexed [I, J, K]."""
    for s, w in enumerate(where):
        if w[0] < 0:
            continue
        v = _face_view(pool, s, axis)  # [k, j, i]
        for K in range(RATIO + (axis == 3)):
            for J in range(RATIO + (axis == 2)):
                for I in range(RATIO + (axis == 1)):
                    acc = np.float32(0)
                    for q in range(RATIO):
                        for p in range(RATIO):
                            fi = RATIO * I + (0 if axis == 1 else p)
                            fj = RATIO * J + (p if axis == 1 else (0 if axis == 2 else q))
                            fk = RATIO * K + (0 if axis == 3 else q)
                            acc = np.float32(acc + v[fk, fj, fi])
                    coarse[RATIO * w[0] + I, RATIO * w[1] + J, RATIO * w[2] + K] = acc / np.float32(16)


def funnel_height(r, h0, depth, width):
    """The surface height at radius r: a Gaussian funnel ``depth`` deep, ``width`` wide."""
    return (h0 - depth * np.exp(-(r / width) ** 2)).astype(np.float32)


def sparse_basin(nb=(4, 4, 4), *, dx: float = 0.05, seed: int = 2001, wall: float = 0.45, height: float = 0.55,
                 funnel: float = 0.25, rings: int = 0, free_every: int = 5, warm: bool = False,
                 swirl: float = 2.0) -> SparseScene:
    """A cylindrical sparse basin of ``nb`` blocks (16^3 fine cells each) a side.

    ``wall`` is the cylinder's radius as a fraction of the box's x width, ``height`` the
    still surface as a fraction of the height above the floor, ``funnel`` the funnel's
    depth as a fraction of that height."""
    nb = tuple(int(b) for b in nb)
    nc = tuple(b * RATIO for b in nb)
    nf = tuple(b * BLOCK for b in nb)
    dx = np.float32(dx)
    cdx = np.float32(RATIO) * dx
    lo = (np.float32(-nf[0] * dx / 2), np.float32(-nf[1] * dx / 2), np.float32(0.0))
    floor_z = np.float32(lo[2] + cdx)
    radius = np.float32(wall * nf[0] * dx)
    top = nf[2] * dx
    h0 = np.float32(floor_z + height * (top - floor_z))
    depth = np.float32(funnel * (h0 - floor_z))
    width = np.float32(0.3 * radius)
    grid = SparseGrid(lo=tuple(float(v) for v in lo), dx=float(dx), nb=nb, radius=float(radius),
                      floor_z=float(floor_z))

    def phi_at(px, py, pz):
        r = np.sqrt(px.astype(np.float64) ** 2 + py.astype(np.float64) ** 2)
        return (pz - funnel_height(r, float(h0), float(depth), float(width))).astype(np.float32)

    # the coarse grid's level set and the blocks the surface passes through
    cx, cy, cz = (_centres(lo[a], cdx, nc[a]) for a in range(3))
    CX, CY, CZ = np.meshgrid(cx, cy, cz, indexing="ij")
    phic = phi_at(CX, CY, CZ)
    csolid = _solid(grid, CX, CY, CZ)
    near = (np.abs(phic) < 1.5 * cdx) & ~csolid
    sign = phic < 0
    for a in range(3):
        flip = sign != np.roll(sign, 1, axis=a)
        idx = [slice(None)] * 3
        idx[a] = 0
        flip[tuple(idx)] = False
        near |= flip & ~csolid
        near |= np.roll(flip, -1, axis=a) & ~csolid
    marks = near.reshape(nb[0], RATIO, nb[1], RATIO, nb[2], RATIO).any(axis=(1, 3, 5))
    for _ in range(rings):
        m = marks.copy()
        for a in range(3):
            for sh in (-1, 1):
                r = np.roll(marks, sh, axis=a)
                idx = [slice(None)] * 3
                idx[a] = 0 if sh == 1 else -1
                r[tuple(idx)] = False
                m |= r
        marks = m
    nblocks = nb[0] * nb[1] * nb[2]
    want = np.flatnonzero(marks.transpose(2, 1, 0).reshape(-1))  # block ids, bi fastest
    slot = np.zeros(nblocks, dtype=np.int32)
    wheres = []
    for b in want:
        if free_every and (len(wheres) + 1) % free_every == 0:
            wheres.append((-1, -1, -1))  # a slot released by an earlier refinement
        wheres.append((b % nb[0], (b // nb[0]) % nb[1], b // (nb[0] * nb[1])))
        slot[b] = len(wheres)
    nslots = len(wheres)
    where = np.array(wheres, dtype=np.int32).reshape(nslots, 3)

    # fine cells of each slot: level set and classes
    lc = np.arange(BCELLS)
    li, lj, lk = lc & 15, (lc >> 4) & 15, lc >> 8
    tf = np.zeros(nslots * BCELLS, dtype=np.uint8)
    phif = np.zeros(nslots * BCELLS, dtype=np.float32)
    for s, w in enumerate(where):
        if w[0] < 0:
            continue
        I, J, K = w[0] * BLOCK + li, w[1] * BLOCK + lj, w[2] * BLOCK + lk
        px = (np.float32(lo[0]) + (I.astype(np.float32) + np.float32(0.5)) * dx).astype(np.float32)
        py = (np.float32(lo[1]) + (J.astype(np.float32) + np.float32(0.5)) * dx).astype(np.float32)
        pz = (np.float32(lo[2]) + (K.astype(np.float32) + np.float32(0.5)) * dx).astype(np.float32)
        ph = phi_at(px, py, pz)
        sl = slice(s * BCELLS, (s + 1) * BCELLS)
        phif[sl] = ph
        tf[sl] = np.where(_solid(grid, px, py, pz), SOLID, np.where(ph < 0, LIQUID, AIR))

    # coarse classes: their own level set outside fine blocks; under them AIR if any fine
    # cell is, else LIQUID if any is, else SOLID; the level set the mean of the 64
    tc = np.where(csolid, SOLID, np.where(phic < 0, LIQUID, AIR)).astype(np.uint8)
    for s, w in enumerate(where):
        if w[0] < 0:
            continue
        t = tf[s * BCELLS:(s + 1) * BCELLS].reshape(BLOCK, BLOCK, BLOCK)  # [k, j, i]
        p = phif[s * BCELLS:(s + 1) * BCELLS].reshape(BLOCK, BLOCK, BLOCK)
        tt = t.reshape(RATIO, RATIO, RATIO, RATIO, RATIO, RATIO)  # [K, c, J, b, I, a]
        air = (tt == AIR).any(axis=(1, 3, 5))
        liq = (tt == LIQUID).any(axis=(1, 3, 5))
        cls = np.where(air, AIR, np.where(liq, LIQUID, SOLID)).astype(np.uint8)  # [K, J, I]
        pm = p.reshape(RATIO, RATIO, RATIO, RATIO, RATIO, RATIO).astype(np.float32).sum(axis=(1, 3, 5),
                                                                                       dtype=np.float32)
        bi, bj, bk = (int(v) * RATIO for v in w)
        tc[bi:bi + RATIO, bj:bj + RATIO, bk:bk + RATIO] = cls.transpose(2, 1, 0)
        phic[bi:bi + RATIO, bj:bj + RATIO, bk:bk + RATIO] = (pm / np.float32(64)).transpose(2, 1, 0)

    # velocities: a swirl about the axis plus noise
    def swirl_at(axis, px, py):
        r2 = px.astype(np.float64) ** 2 + py.astype(np.float64) ** 2 + 1e-6
        s = swirl * np.exp(-r2 / (2.0 * float(width) ** 2)) / np.sqrt(r2) * float(width)
        return (-s * py if axis == 1 else (s * px if axis == 2 else 0.0 * px)).astype(np.float32)

    def fine_faces(axis, aid):
        out = uniform(seed, aid, nslots * BFACES, -0.5, 0.5)
        f = np.arange(BFACES)
        if axis == 1:
            i, j, k = f % 17, (f // 17) & 15, f // 272
        elif axis == 2:
            i, j, k = f & 15, (f >> 4) % 17, (f >> 4) // 17
        else:
            i, j, k = f & 15, (f >> 4) & 15, f >> 8
        for s, w in enumerate(where):
            sl = slice(s * BFACES, (s + 1) * BFACES)
            if w[0] < 0:
                out[sl] = 0
                continue
            off = [0.5, 0.5, 0.5]
            off[axis - 1] = 0.0
            px = (np.float32(lo[0]) + ((w[0] * BLOCK + i) + off[0]) * dx).astype(np.float32)
            py = (np.float32(lo[1]) + ((w[1] * BLOCK + j) + off[1]) * dx).astype(np.float32)
            out[sl] += swirl_at(axis, px, py)
        return out

    def coarse_faces(axis, aid):
        n = list(nc)
        n[axis - 1] += 1
        off = [0.5, 0.5, 0.5]
        off[axis - 1] = 0.0
        gx = (np.float32(lo[0]) + (np.arange(n[0]) + off[0]) * cdx).astype(np.float32)
        gy = (np.float32(lo[1]) + (np.arange(n[1]) + off[1]) * cdx).astype(np.float32)
        X, Y, _ = np.meshgrid(gx, gy, np.zeros(n[2], np.float32), indexing="ij")
        noise = uniform(seed, aid, int(np.prod(n)), -0.5, 0.5).reshape(n[::-1]).transpose(2, 1, 0)
        return (swirl_at(axis, X, Y) + noise).astype(np.float32)

    uf, vf, wf = fine_faces(1, 11), fine_faces(2, 12), fine_faces(3, 13)
    uc, vc, wc = coarse_faces(1, 21), coarse_faces(2, 22), coarse_faces(3, 23)
    for axis, ff, cf in ((1, uf, uc), (2, vf, vc), (3, wf, wc)):
        sync_planes(slot, where, nb, axis, ff)
        restrict_faces(where, axis, ff, cf)
    Pf = np.zeros(nslots * BCELLS, dtype=np.float32)
    Pc = np.zeros(nc, dtype=np.float32)
    if warm:
        Pf[:] = np.where(tf == LIQUID, uniform(seed, 31, Pf.size, 0.0, 0.01), 0).astype(np.float32)
        Pc[:] = np.where(tc == LIQUID, uniform(seed, 32, Pc.size, 0.0, 0.01).reshape(nc[::-1]).transpose(2, 1, 0),
                         0).astype(np.float32)

    def F(a):  # coarse arrays are stored column-major: flatten in Fortran order
        return np.ascontiguousarray(a.reshape(-1, order="F"))

    return SparseScene(
        grid=grid, slot=slot, where=where, nslots=nslots, tf=tf, tc=F(tc), phif=phif, phic=F(phic), Pf=Pf,
        Pc=F(Pc), uf=uf, vf=vf, wf=wf, uc=F(uc), vc=F(vc), wc=F(wc),
        fuf=np.zeros(nslots * BFACES, np.uint8), fvf=np.zeros(nslots * BFACES, np.uint8),
        fwf=np.zeros(nslots * BFACES, np.uint8), fuc=np.zeros(uc.size, np.uint8), fvc=np.zeros(vc.size, np.uint8),
        fwc=np.zeros(wc.size, np.uint8), seed=seed)


def charybdis(nb=(32, 32, 16), seed: int = 2016) -> SparseScene:
    """The sparse benchmark basin: 32 x 32 x 16 blocks (512 x 512 x 256 fine-cell box,
    coarse grid 128 x 128 x 64), a whirlpool funnel through a band of fine blocks."""
    return sparse_basin(nb, seed=seed, funnel=0.45, rings=1, free_every=0, warm=True)
