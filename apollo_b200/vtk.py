"""VTK output of a solution frame, in place of Apollo's ApSolver::writeData
(src/solvers/apsolver.cc:404-419), which hands the state vector to PETSc's VTK
viewer as ``<runName>_<frame>.vtu``.

The file is a VTK XML UnstructuredGrid: the mesh vertices, the triangles, and
as cell data

* ``solution``: each element's state in Apollo's layout (node-major, then
  field: Np * m components per cell), as PETSc's viewer writes a cell section;
* one array per field with the element's average (the reference element's
  averaging weights: half the column sums of its mass matrix), for plotting.

Arrays are written in VTK's inline "binary" format (base64 of a 64-bit byte
count followed by the little-endian data).  ``read_vtu`` reads such files back.
"""
from __future__ import annotations

import base64
import os
import xml.etree.ElementTree as ET

import numpy as np

from .mesh import Mesh

FIELD_NAMES = {
    1: ("q",),
    3: ("Ez", "Bx", "By"),
    4: ("rho", "rhou", "rhov", "E"),
    5: ("rho", "rhou", "rhov", "rhow", "E"),
    8: ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "phi", "psi"),
}


def _b64(a: np.ndarray) -> str:
    raw = np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<"), copy=False).tobytes()
    return base64.b64encode(np.uint64(len(raw)).tobytes() + raw).decode("ascii")


def _data_array(parent, name, a: np.ndarray, ncomp: int = 1):
    vt = {np.dtype(np.float64): "Float64", np.dtype(np.int64): "Int64", np.dtype(np.uint8): "UInt8"}[a.dtype]
    e = ET.SubElement(parent, "DataArray", type=vt, Name=name, NumberOfComponents=str(ncomp), format="binary")
    e.text = _b64(a.ravel())
    return e


def write_vtu(path: str, mesh: Mesh, U: np.ndarray, averages=None, field_names=None, time: float | None = None):
    """Write one frame.  U: float64 [K][Np][m] (Apollo's layout); averages:
    the nodal averaging weights [Np] (``NodalDG2d.averaging_weights()``), or
    None to skip the per-field averages."""
    U = np.ascontiguousarray(U, dtype=np.float64)
    K, Np, m = U.shape
    assert K == mesh.K
    names = field_names or FIELD_NAMES.get(m, tuple(f"q{i}" for i in range(m)))
    root = ET.Element("VTKFile", type="UnstructuredGrid", version="1.0", byte_order="LittleEndian",
                      header_type="UInt64")
    grid = ET.SubElement(root, "UnstructuredGrid")
    if time is not None:
        fd = ET.SubElement(grid, "FieldData")
        _data_array(fd, "TIME", np.array([time], dtype=np.float64))
    piece = ET.SubElement(grid, "Piece", NumberOfPoints=str(mesh.nverts), NumberOfCells=str(K))
    pts = ET.SubElement(piece, "Points")
    xyz = np.stack([mesh.vx, mesh.vy, np.zeros_like(mesh.vx)], axis=1)
    _data_array(pts, "Points", xyz.astype(np.float64), 3)
    cells = ET.SubElement(piece, "Cells")
    _data_array(cells, "connectivity", mesh.etov.astype(np.int64))
    _data_array(cells, "offsets", (3 * np.arange(1, K + 1)).astype(np.int64))
    _data_array(cells, "types", np.full(K, 5, dtype=np.uint8))  # VTK_TRIANGLE
    cd = ET.SubElement(piece, "CellData", Scalars="solution")
    _data_array(cd, "solution", U.reshape(K, Np * m), Np * m)
    if averages is not None:
        w = np.asarray(averages, dtype=np.float64)
        avg = np.einsum("n,knm->km", w, U)
        for i, nm in enumerate(names):
            _data_array(cd, nm, np.ascontiguousarray(avg[:, i]))
    ET.ElementTree(root).write(path, xml_declaration=True, encoding="utf-8")


def write_frame(run_name: str, frame: int, mesh: Mesh, U: np.ndarray, averages=None, time: float | None = None,
                directory: str = ".") -> str:
    """Apollo's frame file name, ``<runName>_<frame>.vtu``; returns the path."""
    path = os.path.join(directory, f"{run_name}_{frame}.vtu")
    write_vtu(path, mesh, U, averages=averages, time=time)
    return path


def read_vtu(path: str) -> dict:
    """The arrays of a file written by ``write_vtu``, by name (points, the
    three cell arrays, and the cell data)."""
    root = ET.parse(path).getroot()
    types = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}
    out = {}
    for e in root.iter("DataArray"):
        raw = base64.b64decode(e.text)
        n = int(np.frombuffer(raw[:8], dtype="<u8")[0])
        a = np.frombuffer(raw[8:8 + n], dtype=np.dtype(types[e.get("type")]).newbyteorder("<"))
        nc = int(e.get("NumberOfComponents", "1"))
        out[e.get("Name")] = a.reshape(-1, nc) if nc > 1 else a
    return out
