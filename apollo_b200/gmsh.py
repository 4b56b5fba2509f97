"""Gmsh 2.2 ASCII meshes: ``read_gmsh`` (the library's reader,
apollo_dg_mesh_read_gmsh) and ``write_gmsh`` (triangles plus tagged boundary
lines, the form Apollo's example inputs use)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .dg import ApolloError, _dp, _ip, load_library
from .mesh import Mesh

def read_gmsh(path: str) -> Mesh:
    """Triangles (counter-clockwise) and face tags from the physical tags of the
    boundary lines (Apollo's "Face Sets" rule; see include/apollo_dg.h)."""
    lib = load_library()
    h = C.c_void_p()
    err = C.create_string_buffer(512)
    code = lib.apollo_dg_mesh_read_gmsh(str(path).encode(), C.byref(h), err, len(err))
    if code:
        raise ApolloError(code, err.value.decode())
    try:
        nv, K = C.c_int(), C.c_int()
        lib.apollo_dg_mesh_info(h, C.byref(nv), C.byref(K))
        vx, vy = np.empty(nv.value), np.empty(nv.value)
        etov = np.empty((K.value, 3), dtype=np.int32)
        tag = np.empty((K.value, 3), dtype=np.int32)
        lib.apollo_dg_mesh_arrays(h, vx.ctypes.data_as(_dp), vy.ctypes.data_as(_dp), etov.ctypes.data_as(_ip),
                                  tag.ctypes.data_as(_ip))
    finally:
        lib.apollo_dg_mesh_destroy(h)
    return Mesh(vx=vx, vy=vy, etov=etov, face_tag=tag, vert_canon=np.arange(nv.value, dtype=np.int32), n=0,
                lo=(float(vx.min()), float(vy.min())), hi=(float(vx.max()), float(vy.max())), periodic=False)


def write_gmsh(mesh: Mesh, path: str, physical_surface: int = 1) -> None:
    """Gmsh 2.2 ASCII: every vertex, one line element per tagged face (physical
    tag = the face tag, elementary tag = the same) and the triangles (physical
    tag ``physical_surface``).  Periodic identifications are not written."""
    tags = np.asarray(mesh.face_tag)
    vn = ((0, 1), (1, 2), (2, 0))
    lines = [(mesh.etov[k, vn[f][0]], mesh.etov[k, vn[f][1]], tags[k, f])
             for k, f in zip(*np.nonzero(tags > 0))]
    with open(path, "w") as fh:
        fh.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n")
        fh.write(f"$Nodes\n{mesh.nverts}\n")
        for i in range(mesh.nverts):
            fh.write(f"{i + 1} {float(mesh.vx[i])!r} {float(mesh.vy[i])!r} 0\n")
        fh.write("$EndNodes\n")
        fh.write(f"$Elements\n{len(lines) + mesh.K}\n")
        e = 1
        for a, b, t in lines:
            fh.write(f"{e} 1 2 {t} {t} {a + 1} {b + 1}\n")
            e += 1
        for k in range(mesh.K):
            a, b, c = mesh.etov[k]
            fh.write(f"{e} 2 2 {physical_surface} {physical_surface} {a + 1} {b + 1} {c + 1}\n")
            e += 1
        fh.write("$EndElements\n")
