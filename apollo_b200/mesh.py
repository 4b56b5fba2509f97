"""Seeded jittered triangulations of a rectangle, the meshes the solver runs on.

A mesh is plain arrays, the form ``apollo_dg_set_mesh`` takes:

* ``vx, vy``      float64 [nverts] vertex coordinates
* ``etov``        int32 [K, 3] counter-clockwise vertex triples; vertex 0 maps to
                  reference (r, s) = (-1, -1), vertex 1 to (1, -1), vertex 2 to
                  (-1, 1), so faces are (v0 v1), (v1 v2), (v2 v0) as in Apollo's
                  face numbering (src/lib/wxnodaldggeometry2d.cc:263)
* ``face_tag``    int32 [K, 3]: 0 = pair with the face sharing both vertices,
                  t > 0 = physical boundary using boundary condition t (1-based,
                  Apollo's ``boundaryConditions[t-1]``)
* ``vert_canon``  int32 [nverts] canonical vertex id used for pairing; periodic
                  meshes identify vertices across opposite sides

Vertices sit on an n x n grid of spacing h = L/(n-1); every grid cell is split
into two triangles along the same diagonal, giving K = 2 (n-1)^2 elements.
Interior vertices are moved by independent uniform offsets in [-a h, a h] in x
and y, drawn from ``numpy.random.default_rng(seed)`` (PCG64) in vertex order.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Mesh:
    vx: np.ndarray
    vy: np.ndarray
    etov: np.ndarray
    face_tag: np.ndarray
    vert_canon: np.ndarray
    n: int
    lo: tuple
    hi: tuple
    periodic: bool

    @property
    def K(self) -> int:
        return int(self.etov.shape[0])

    @property
    def nverts(self) -> int:
        return int(self.vx.shape[0])


def jittered_square(n: int, lo=(0.0, 0.0), hi=(1.0, 1.0), jitter: float = 0.2, seed: int = 0,
                    periodic: bool = True, wall_tag: int = 1, ny: int | None = None) -> Mesh:
    """n x ny vertex grid (ny = n by default) on [lo, hi], 2 (n-1)(ny-1)
    triangles, interior vertices jittered.

    With ``periodic`` the boundary faces pair with the faces on the opposite
    side; otherwise they carry ``wall_tag``.
    """
    ny = n if ny is None else ny
    if n < 3 or ny < 3:
        raise ValueError("need at least a 3 x 3 vertex grid")
    x0, y0 = float(lo[0]), float(lo[1])
    x1, y1 = float(hi[0]), float(hi[1])
    hx, hy = (x1 - x0) / (n - 1), (y1 - y0) / (ny - 1)
    ii, jj = np.meshgrid(np.arange(n), np.arange(ny), indexing="xy")
    ii = ii.ravel()
    jj = jj.ravel()
    vx = x0 + ii * hx
    vy = y0 + jj * hy
    # exact end coordinates on the boundary lines
    vx[ii == n - 1] = x1
    vy[jj == ny - 1] = y1
    rng = np.random.default_rng(seed)
    offs = rng.uniform(-jitter, jitter, size=(n * ny, 2))
    interior = (ii > 0) & (ii < n - 1) & (jj > 0) & (jj < ny - 1)
    vx = np.where(interior, vx + offs[:, 0] * hx, vx)
    vy = np.where(interior, vy + offs[:, 1] * hy, vy)

    ci, cj = np.meshgrid(np.arange(n - 1), np.arange(ny - 1), indexing="xy")
    ci = ci.ravel()
    cj = cj.ravel()
    v00 = cj * n + ci
    v10 = v00 + 1
    v01 = v00 + n
    v11 = v01 + 1
    etov = np.empty((2 * (n - 1) * (ny - 1), 3), dtype=np.int32)
    etov[0::2] = np.stack([v00, v10, v11], axis=1)
    etov[1::2] = np.stack([v00, v11, v01], axis=1)

    if periodic:
        canon = ((jj % (ny - 1)) * n + (ii % (n - 1))).astype(np.int32)
        face_tag = np.zeros_like(etov)
    else:
        canon = np.arange(n * ny, dtype=np.int32)
        face_tag = np.zeros_like(etov)
        onb = (ii == 0) | (ii == n - 1) | (jj == 0) | (jj == ny - 1)
        for f, (a, b) in enumerate(((0, 1), (1, 2), (2, 0))):
            va, vb = etov[:, a], etov[:, b]
            same_x = (ii[va] == ii[vb]) & ((ii[va] == 0) | (ii[va] == n - 1))
            same_y = (jj[va] == jj[vb]) & ((jj[va] == 0) | (jj[va] == ny - 1))
            face_tag[:, f] = np.where(onb[va] & onb[vb] & (same_x | same_y), wall_tag, 0)
    return Mesh(vx=np.ascontiguousarray(vx, dtype=np.float64), vy=np.ascontiguousarray(vy, dtype=np.float64),
                etov=etov, face_tag=face_tag.astype(np.int32), vert_canon=canon, n=n,
                lo=(x0, y0), hi=(x1, y1), periodic=periodic)


def grid_for_elements(K_target: int) -> int:
    """Vertex-grid size n whose 2 (n-1)^2 elements are nearest K_target."""
    m = max(2, int(round((K_target / 2.0) ** 0.5)))
    return m + 1
