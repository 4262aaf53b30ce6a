"""Seeded synthetic basins: the inputs a FlipBasin hands to ``project!``.

The reference builds these arrays with its own scene code (``FlipGrid``,
``classify!``, ``forces!`` -> ``solidify!``); no public dataset exists for the path.
This module makes the same arrays for a cylindrical basin on a box grid:

* geometry as ``FlipGrid`` (src/flip.jl:39-66): cell centres at ``lo + (i+1/2) dx``,
  a cell is SOLID when its centre is outside the cylinder or under the floor;
* ``phi`` the free-surface level set, ``types`` LIQUID where ``phi < 0`` else AIR
  (``classify_kernel!``, src/flip.jl:682-686);
* face velocities iid uniform[-1, 1) m/s from a counter-based generator
  (splitmix64 of seed, array id and linear index), optionally plus a Rankine
  vortex and edge eddies, then zero on walled faces (``solidify!``,
  src/flip.jl:778-807), as ``forces!`` leaves them before every projection.

All arithmetic that decides a cell's class is Float32, as in the reference.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

SOLID, LIQUID, AIR = 0, 1, 2

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def _mix64(z: np.ndarray) -> np.ndarray:
    """splitmix64's finaliser (Steele, Lea & Flood 2014), on uint64 arrays."""
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform(seed: int, array_id: int, count: int, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    """``count`` float32 values uniform in [lo, hi): value n = f(seed, array_id, n)."""
    with np.errstate(over="ignore"):
        key = _mix64(np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + _GOLDEN * np.uint64(array_id + 1))
        idx = np.arange(1, count + 1, dtype=np.uint64)
        bits = _mix64(key + _GOLDEN * idx) >> np.uint64(40)
    unit = bits.astype(np.float64) * (1.0 / (1 << 24))
    return (lo + (hi - lo) * unit).astype(np.float32)


def levels_for(n) -> int:
    """``FlipGrid``'s level count (src/flip.jl:53-61): the fewest levels (at least 2) whose
    coarsest grid, ``n / 2^(levels-1)``, has at most 1024 cells."""
    levels = 2
    while True:
        m = 1 << (levels - 1)
        if any(x % m for x in n):
            raise ValueError(f"grid {tuple(n)} is not a multiple of {m}; FlipGrid pads it to one")
        if (n[0] // m) * (n[1] // m) * (n[2] // m) <= 1024:
            return levels
        levels += 1


@dataclasses.dataclass
class Grid:
    """``FlipGrid`` (src/flip.jl:39-46)."""

    lo: tuple
    dx: float
    n: tuple
    radius: float
    floor: float
    levels: int

    @property
    def ncells(self) -> int:
        return self.n[0] * self.n[1] * self.n[2]

    def face_shape(self, axis: int) -> tuple:
        """Column-major dims of the face array along ``axis`` (u: (nx+1, ny, nz), ...)."""
        return tuple(self.n[a] + (1 if a == axis else 0) for a in range(3))


@dataclasses.dataclass
class Basin:
    """The projection's inputs, as flat column-major arrays (i fastest)."""

    grid: Grid
    types: np.ndarray  # uint8, ncells
    phi: np.ndarray  # float32, ncells
    u: np.ndarray  # float32, (nx+1)*ny*nz
    v: np.ndarray
    w: np.ndarray
    seed: int
    name: str = ""

    def copy(self) -> "Basin":
        return dataclasses.replace(self, types=self.types.copy(), phi=self.phi.copy(),
                                   u=self.u.copy(), v=self.v.copy(), w=self.w.copy())

    @property
    def liquid_fraction(self) -> float:
        return float(np.count_nonzero(self.types == LIQUID)) / self.types.size


def _centres(grid: Grid, axis: int, count: int, offset: float) -> np.ndarray:
    """Float32 positions ``lo + (i + offset) dx`` along ``axis``, as ``cellcentre``/``nodepos``."""
    i = np.arange(count, dtype=np.float32)
    return (np.float32(grid.lo[axis]) + (i + np.float32(offset)) * np.float32(grid.dx)).astype(np.float32)


def solid_cells(grid: Grid) -> np.ndarray:
    """``issolidcell`` for every cell (src/flip.jl:64-66), as a bool array shaped (nz, ny, nx)."""
    x = _centres(grid, 0, grid.n[0], 0.5)
    y = _centres(grid, 1, grid.n[1], 0.5)
    z = _centres(grid, 2, grid.n[2], 0.5)
    r2 = (x[None, :] * x[None, :] + y[:, None] * y[:, None]).astype(np.float32)
    outside = r2 > np.float32(grid.radius) * np.float32(grid.radius)
    below = z < np.float32(grid.floor)
    return outside[None, :, :] | below[:, None, None]


def solidify(grid: Grid, arr: np.ndarray, axis: int, solid: np.ndarray | None = None) -> None:
    """Zero every walled face in place (``walled``/``solid_kernel!``, src/flip.jl:777-789):
    a face on the box edge, or with a SOLID cell on either side."""
    if solid is None:
        solid = solid_cells(grid)
    shape = grid.face_shape(axis)[::-1]  # (nz, ny, nx) view of column-major data
    a = arr.reshape(shape)
    walled = np.ones(shape, dtype=bool)
    if axis == 0:
        walled[:, :, 1:-1] = solid[:, :, :-1] | solid[:, :, 1:]
    elif axis == 1:
        walled[:, 1:-1, :] = solid[:, :-1, :] | solid[:, 1:, :]
    else:
        walled[1:-1, :, :] = solid[:-1, :, :] | solid[1:, :, :]
    a[walled] = 0.0


def rankine(r: np.ndarray, circulation: float, core: float) -> np.ndarray:
    """Azimuthal speed of a Rankine vortex: Gamma r / (2 pi c^2) inside the core, Gamma / (2 pi r) out."""
    r = np.asarray(r, dtype=np.float64)
    inside = circulation * r / (2.0 * math.pi * core * core)
    outside = circulation / (2.0 * math.pi * np.maximum(r, 1e-12))
    return np.where(r < core, inside, outside)


def rankine_surface(r: np.ndarray, circulation: float, core: float, g: float = 9.81) -> np.ndarray:
    """Cyclostrophic free surface of a Rankine vortex (the integral ``balanced`` takes,
    src/sea.jl:48-58, for this profile): -G^2/(8 pi^2 g r^2) outside the core,
    -G^2/(4 pi^2 g c^2) + G^2 r^2/(8 pi^2 g c^4) inside."""
    r = np.asarray(r, dtype=np.float64)
    k = circulation * circulation / (8.0 * math.pi * math.pi * g)
    outside = -k / np.maximum(r * r, 1e-12)
    inside = -2.0 * k / (core * core) + k * r * r / core ** 4
    return np.where(r < core, inside, outside)


def box_basin(n, *, dx: float = 0.05, seed: int = 1001, wall: float = 0.45, height: float = 0.6,
              vortex: float | None = None, core: float = 2.5, depression: bool = False,
              eddy: float = 0.0, eddy_band: float = 0.9, speed: float = 1.0, name: str = "") -> Basin:
    """A cylindrical basin in an ``n`` box (``n`` an int for a cube, or 3 ints).

    ``wall`` is the cylinder radius over the box's x edge, ``height`` the still water
    depth over the box height. ``vortex`` adds a Rankine vortex of that circulation
    (m^2/s, core ``core`` m) to u and v; ``depression`` lowers the free surface by its
    cyclostrophic profile; ``eddy`` adds uniform[-eddy, eddy) m/s noise to all three
    components outside ``eddy_band`` of the radius. Faces are walled off last.
    """
    if isinstance(n, int):
        n = (n, n, n)
    n = tuple(int(x) for x in n)
    grid = Grid(lo=(float(np.float32(-n[0] * dx / 2)), float(np.float32(-n[1] * dx / 2)), 0.0),
                dx=float(np.float32(dx)), n=n, radius=float(np.float32(wall * n[0] * dx)), floor=0.0,
                levels=levels_for(n))
    solid = solid_cells(grid)
    x = _centres(grid, 0, n[0], 0.5)
    y = _centres(grid, 1, n[1], 0.5)
    z = _centres(grid, 2, n[2], 0.5)
    h = np.float32(height * n[2] * dx)
    if depression and vortex:
        r = np.sqrt(x[None, :].astype(np.float64) ** 2 + y[:, None].astype(np.float64) ** 2)
        surf = (h + rankine_surface(r, vortex, core)).astype(np.float32)  # (ny, nx)
        phi = (z[:, None, None] - surf[None, :, :]).astype(np.float32)
    else:
        phi = np.broadcast_to((z - h).astype(np.float32)[:, None, None], (n[2], n[1], n[0])).copy()
    types = np.where(solid, SOLID, np.where(phi < 0, LIQUID, AIR)).astype(np.uint8)

    faces = []
    for axis in range(3):
        shape = grid.face_shape(axis)
        count = shape[0] * shape[1] * shape[2]
        f = uniform(seed, axis, count, -speed, speed).reshape(shape[::-1])
        if vortex or eddy:
            fx = _centres(grid, 0, shape[0], 0.0 if axis == 0 else 0.5).astype(np.float64)
            fy = _centres(grid, 1, shape[1], 0.0 if axis == 1 else 0.5).astype(np.float64)
            r = np.sqrt(fx[None, :] ** 2 + fy[:, None] ** 2)  # (ny', nx')
            extra = np.zeros(r.shape, dtype=np.float64)
            if vortex and axis < 2:
                ut = rankine(r, vortex, core)
                comp = (-fy[:, None] if axis == 0 else fx[None, :]) / np.maximum(r, 1e-12)
                extra = ut * comp
            f = (f.astype(np.float64) + extra[None, :, :]).astype(np.float32)
            if eddy:
                noise = uniform(seed, 10 + axis, count, -eddy, eddy).reshape(shape[::-1])
                band = (r > eddy_band * grid.radius)[None, :, :]
                f = np.where(band, f + noise, f).astype(np.float32)
        f = np.ascontiguousarray(f).reshape(-1)
        solidify(grid, f, axis, solid)
        faces.append(f)
    return Basin(grid=grid, types=types.reshape(-1), phi=phi.reshape(-1), u=faces[0], v=faces[1],
                 w=faces[2], seed=seed, name=name or f"box{n[0]}x{n[1]}x{n[2]}")


# The workloads, by name: sizes and seeds as the benchmark configurations state them.
BATCH_EDGES = (48, 64, 96, 128)


def batch_basins(count: int = 48, seed: int = 1002) -> list:
    """The batched workload: ``count`` independent cubic basins, edge drawn per basin from
    {48, 64, 96, 128}, still-water height fraction uniform[0.3, 0.8], wall radius fraction
    uniform[0.35, 0.48], faces uniform[-1, 1) m/s; everything from the one ``seed`` (basin
    b's face seed is seed * 1000 + b)."""
    out = []
    for b in range(count):
        r = uniform(seed, 900 + b, 3, 0.0, 1.0).astype(np.float64)  # three draws in [0, 1)
        edge = BATCH_EDGES[min(int(r[0] * len(BATCH_EDGES)), len(BATCH_EDGES) - 1)]
        height = 0.3 + 0.5 * float(r[1])
        wall = 0.35 + 0.13 * float(r[2])
        out.append(box_basin(edge, seed=seed * 1000 + b, wall=wall, height=height, name=f"batch{b}"))
    return out


def config_basin(name: str) -> Basin:
    """``plain64``: 64^3 (seed 1000); ``whirl256``: 256^3 plus a Rankine vortex
    (Gamma = 225 m^2/s, core 2.5 m; seed 1001); ``whirlpool384``: 384x384x256, surface
    0.7 deep lowered by the vortex, eddies in the outer tenth (seed 1004)."""
    if name == "plain64":
        return box_basin(64, seed=1000, name=name)
    if name == "whirl256":
        return box_basin(256, seed=1001, vortex=225.0, core=2.5, name=name)
    if name == "whirlpool384":
        return box_basin((384, 384, 256), seed=1004, height=0.7, vortex=225.0, core=2.5, depression=True,
                         eddy=0.5, eddy_band=0.9, name=name)
    if name.startswith("box"):
        return box_basin(int(name[3:]), seed=1000 + int(name[3:]), name=name)
    raise KeyError(name)
