"""Generate the golden pressure fixtures: exact solutions of the reference's linear system.

    python tests/golden/make_golden.py

The reference's own tests hold no values for this path, so these fixtures pin the oracle
and the CUDA path to the reference's *equations* instead: the ghost-fluid Poisson system
of src/flip.jl:809-836 (rows on LIQUID cells: diag P_i - sum over LIQUID neighbours of
P_n = b_i, diag = #LIQUID neighbours + sum over AIR neighbours of 1/theta, walls and the
box edge contribute nothing; b = -dx div u + dx^2 gamma), assembled here from the scene
arrays with scipy and solved directly (sparse LU), independently of oracle/ and libmpp.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "maelstrom.jl_b200"))

from mpp import scene  # noqa: E402

CASES = {
    # name: (basin kwargs, gamma)
    "box16": (dict(n=16, seed=1016), 0.0),
    "box32": (dict(n=32, seed=1032), 0.0),
    "box32_gamma": (dict(n=32, seed=2032, height=0.45, wall=0.4), 0.05),
    "box16x16x32": (dict(n=(16, 16, 32), seed=3016, height=0.7), 0.0),
}


def assemble(basin, gamma):
    """A (on LIQUID cells) and b, in float64, from the reference's definitions."""
    g = basin.grid
    n1, n2, n3 = g.n
    t = basin.types.reshape(n3, n2, n1)
    phi = basin.phi.reshape(n3, n2, n1).astype(np.float64)
    liquid = t == scene.LIQUID
    idx = -np.ones(t.shape, dtype=np.int64)
    idx[liquid] = np.arange(int(liquid.sum()))
    rows, cols, vals = [], [], []
    diag = np.zeros(int(liquid.sum()))
    K, J, I = np.nonzero(liquid)
    for (dk, dj, di) in ((0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 0), (-1, 0, 0)):
        kk, jj, ii = K + dk, J + dj, I + di
        inside = (ii >= 0) & (ii < n1) & (jj >= 0) & (jj < n2) & (kk >= 0) & (kk < n3)
        tn = np.full(K.shape, scene.SOLID)
        tn[inside] = t[kk[inside], jj[inside], ii[inside]]
        me = idx[K, J, I]
        nl = tn == scene.LIQUID
        diag[me[nl]] += 1.0
        rows.append(me[nl])
        cols.append(idx[kk[nl], jj[nl], ii[nl]])
        vals.append(-np.ones(int(nl.sum())))
        na = tn == scene.AIR
        pi = phi[K[na], J[na], I[na]]
        pj = phi[kk[na], jj[na], ii[na]]
        theta = np.clip(pi / (pi - pj), 0.01, 1.0)
        np.add.at(diag, me[na], 1.0 / theta)
    rows.append(np.arange(diag.size))
    cols.append(np.arange(diag.size))
    vals.append(diag)
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(diag.size, diag.size))
    u = basin.u.reshape(n3, n2, n1 + 1).astype(np.float64)
    v = basin.v.reshape(n3, n2 + 1, n1).astype(np.float64)
    w = basin.w.reshape(n3 + 1, n2, n1).astype(np.float64)
    div = (u[:, :, 1:] - u[:, :, :-1]) + (v[:, 1:, :] - v[:, :-1, :]) + (w[1:, :, :] - w[:-1, :, :])
    dx = float(g.dx)
    b = np.where(liquid, -dx * div + dx * dx * gamma, 0.0)
    return A, b.reshape(-1), liquid.reshape(-1)


def scene_digest(basin) -> str:
    h = hashlib.sha256()
    for a in (basin.types, basin.phi, basin.u, basin.v, basin.w):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def build_case(name):
    kw, gamma = CASES[name]
    basin = scene.box_basin(**kw)
    A, b, liquid = assemble(basin, gamma)
    x = spla.spsolve(A.tocsc(), b[liquid])
    P = np.zeros(basin.grid.ncells)
    P[liquid] = x
    return basin, b, P, gamma


def main():
    for name in CASES:
        basin, b, P, gamma = build_case(name)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, b=b, P=P, gamma=gamma, digest=scene_digest(basin))
        print(name, basin.grid.n, "liquid", int((basin.types == scene.LIQUID).sum()), "|P|", np.linalg.norm(P), path)


if __name__ == "__main__":
    main()
