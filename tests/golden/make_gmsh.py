"""Generate tests/golden/square_delaunay.msh: an unstructured Gmsh 2.2 mesh of
[0,10]^2 (Delaunay triangulation of seeded points: 13 points on each side,
a jittered 11 x 11 interior lattice), bottom/top edges tagged 1, left/right
edges tagged 2.

    python tests/golden/make_gmsh.py
"""
from __future__ import annotations

import os
import sys

import numpy as np
from scipy.spatial import Delaunay

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from apollo_b200.gmsh import write_gmsh  # noqa: E402
from apollo_b200.mesh import Mesh  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def main(path=os.path.join(HERE, "square_delaunay.msh"), L=10.0, nb=13, ni=11, seed=11):
    rng = np.random.default_rng(seed)
    s = np.linspace(0.0, L, nb)
    side = np.concatenate([np.stack([s, np.zeros(nb)], 1), np.stack([s, np.full(nb, L)], 1),
                           np.stack([np.zeros(nb - 2), s[1:-1]], 1), np.stack([np.full(nb - 2, L), s[1:-1]], 1)])
    h = L / (ni + 1)
    g = (np.arange(ni) + 1) * h
    gx, gy = np.meshgrid(g, g)
    inner = np.stack([gx.ravel(), gy.ravel()], 1) + rng.uniform(-0.3 * h, 0.3 * h, size=(ni * ni, 2))
    pts = np.concatenate([side, inner])
    tri = Delaunay(pts).simplices.astype(np.int32)
    # counter-clockwise
    a, b, c = pts[tri[:, 0]], pts[tri[:, 1]], pts[tri[:, 2]]
    cw = (b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (c[:, 0] - a[:, 0]) * (b[:, 1] - a[:, 1]) < 0
    tri[cw] = tri[cw][:, [0, 2, 1]]
    tag = np.zeros_like(tri)
    eps = 1e-12
    for f, (i, j) in enumerate(((0, 1), (1, 2), (2, 0))):
        p, q = pts[tri[:, i]], pts[tri[:, j]]
        horiz = (np.abs(p[:, 1] - q[:, 1]) < eps) & ((np.abs(p[:, 1]) < eps) | (np.abs(p[:, 1] - L) < eps))
        vert = (np.abs(p[:, 0] - q[:, 0]) < eps) & ((np.abs(p[:, 0]) < eps) | (np.abs(p[:, 0] - L) < eps))
        tag[:, f] = np.where(horiz, 1, np.where(vert, 2, 0))
    mesh = Mesh(vx=pts[:, 0].copy(), vy=pts[:, 1].copy(), etov=tri, face_tag=tag,
                vert_canon=np.arange(len(pts), dtype=np.int32), n=0, lo=(0, 0), hi=(L, L), periodic=False)
    write_gmsh(mesh, path)
    return mesh


if __name__ == "__main__":
    m = main()
    print(m.nverts, m.K, np.bincount(m.face_tag.ravel()))
