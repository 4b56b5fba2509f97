"""Gmsh 2.2 reader (apollo_dg_mesh_read_gmsh): round trips, the face-tag rule
of Apollo's "Face Sets" handling, malformed input, and Apollo's own example
meshes where the reference tree is present."""
import glob
import os

import numpy as np
import pytest

from apollo_b200 import ApolloError, read_gmsh, write_gmsh
from apollo_b200.mesh import jittered_square
from golden_cases import load

HERE = os.path.dirname(os.path.abspath(__file__))
from oracle.oracle import reference_src

REF_EXAMPLES = os.path.join(reference_src(), "..", "examples", "unstructuredDG")


def test_round_trip_keeps_mesh_and_side_tags(tmp_path):
    m = jittered_square(9, (0.0, 0.0), (2.0, 1.0), seed=4, periodic=False, wall_tag=1)
    # a tag per side: bottom 1, right 2, top 3, left 4
    tag = np.zeros_like(m.face_tag)
    vn = ((0, 1), (1, 2), (2, 0))
    for f, (a, b) in enumerate(vn):
        xa, ya, xb, yb = m.vx[m.etov[:, a]], m.vy[m.etov[:, a]], m.vx[m.etov[:, b]], m.vy[m.etov[:, b]]
        tag[:, f] = np.select([(ya == 0) & (yb == 0), (xa == 2) & (xb == 2), (ya == 1) & (yb == 1),
                               (xa == 0) & (xb == 0)], [1, 2, 3, 4], 0)
    assert np.array_equal(tag > 0, m.face_tag > 0)
    m.face_tag = tag.astype(np.int32)
    path = str(tmp_path / "m.msh")
    write_gmsh(m, path)
    r = read_gmsh(path)
    np.testing.assert_array_equal(r.vx, m.vx)
    np.testing.assert_array_equal(r.vy, m.vy)
    np.testing.assert_array_equal(r.etov, m.etov)
    np.testing.assert_array_equal(r.face_tag, m.face_tag)


TINY = """$MeshFormat
2.2 0 8
$EndMeshFormat
$PhysicalNames
2
1 7 "wall"
2 9 "fluid"
$EndPhysicalNames
$Nodes
5
10 0 0 0
20 1 0 0
30 1 1 0
40 0 1 0
50 0.5 0.5 0
$EndNodes
$Elements
8
1 15 2 0 1 10
2 1 2 7 1 10 20
3 1 2 8 2 20 30
4 1 2 7 3 30 40
5 2 2 9 5 10 20 50
6 2 2 9 5 20 30 50
7 2 2 9 5 40 30 50
8 2 2 9 5 10 50 40
$EndElements
$Periodic
0
$EndPeriodic
"""


def test_tiny_file_ids_orientation_and_tags(tmp_path):
    p = tmp_path / "tiny.msh"
    p.write_text(TINY)
    m = read_gmsh(str(p))
    assert (m.nverts, m.K) == (5, 4)
    np.testing.assert_array_equal(m.vx, [0, 1, 1, 0, 0.5])
    # element 7 was clockwise (40 30 50): stored as 40 50 30
    np.testing.assert_array_equal(m.etov, [[0, 1, 4], [1, 2, 4], [3, 4, 2], [0, 4, 3]])
    # bottom tagged 7, right 8, top 7; the left side (no line element) is
    # unpaired in an element without labels: tag 1 (Apollo's default)
    np.testing.assert_array_equal(m.face_tag, [[7, 0, 0], [8, 0, 0], [0, 0, 7], [0, 0, 1]])


def test_unlabelled_face_takes_its_elements_label(tmp_path):
    """One triangle, two of its edges labelled 5 and 6, the third unlabelled
    and also unpaired: it takes the element's last labelled face's tag."""
    txt = ("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n3\n1 0 0 0\n2 1 0 0\n3 0 1 0\n$EndNodes\n"
           "$Elements\n3\n1 1 1 5 1 2\n2 1 1 6 2 3\n3 2 1 1 1 2 3\n$EndElements\n")
    p = tmp_path / "one.msh"
    p.write_text(txt)
    np.testing.assert_array_equal(read_gmsh(str(p)).face_tag, [[5, 6, 6]])


@pytest.mark.parametrize("body, why", [
    ("$MeshFormat\n2.2 1 8\n$EndMeshFormat\n", "binary"),
    ("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n", "2.x"),
    ("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n3\n1 0 0 0\n2 1 0 0\n$EndNodes\n", "truncated"),
    ("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n4\n1 0 0 0\n2 1 0 0\n3 1 1 0\n4 0 1 0\n$EndNodes\n"
     "$Elements\n1\n1 3 2 1 1 1 2 3 4\n$EndElements\n", "triangles"),
    ("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n3\n1 0 0 0\n2 1 0 0\n3 0 1 0\n$EndNodes\n"
     "$Elements\n1\n1 2 0 1 2 9\n$EndElements\n", "unknown node"),
    ("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n3\n1 0 0 0\n2 1 0 0\n3 2 0 0\n$EndNodes\n"
     "$Elements\n1\n1 2 0 1 2 3\n$EndElements\n", "degenerate"),
])
def test_malformed_input_is_refused(tmp_path, body, why):
    p = tmp_path / "bad.msh"
    p.write_text(body)
    with pytest.raises(ApolloError, match=why):
        read_gmsh(str(p))
    with pytest.raises(ApolloError, match="cannot open"):
        read_gmsh(str(tmp_path / "missing.msh"))


def test_fixture_reads_as_the_golden_case():
    g = load("euler_gmsh_N3")
    m = read_gmsh(os.path.join(HERE, "golden", "square_delaunay.msh"))
    np.testing.assert_array_equal(m.etov, g["etov"])
    np.testing.assert_array_equal(m.face_tag, g["face_tag"])
    np.testing.assert_array_equal(m.vx, g["vx"])
    assert set(np.unique(m.face_tag)) == {0, 1, 2}


def _boundary_lines(path):
    """Line elements of a Gmsh 2.2 file (tags, nodes), read as text."""
    out, inside = [], False
    with open(path) as fh:
        for ln in fh:
            ln = ln.strip()
            if ln == "$Elements":
                inside = True
                next(fh)
                continue
            if ln == "$EndElements":
                break
            if inside:
                w = ln.split()
                if w[1] == "1":
                    out.append(int(w[3]))
    return out


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="Apollo's example inputs are not present")
def test_apollo_example_meshes(oracle_lib):
    files = sorted(glob.glob(os.path.join(REF_EXAMPLES, "euler", "*", "*.msh")))
    assert files
    for f in files:
        m = read_gmsh(f)
        lines = _boundary_lines(f)
        edges = np.sort(np.stack([m.etov[:, [0, 1, 2]], m.etov[:, [1, 2, 0]]], -1), -1).reshape(-1, 2)
        _, inv, cnt = np.unique(edges, axis=0, return_inverse=True, return_counts=True)
        unpaired = (cnt[inv.ravel()] == 1).reshape(-1, 3)
        # exactly the unpaired faces carry a tag; with boundary lines in the
        # file, one line per unpaired face and only their tags
        np.testing.assert_array_equal(m.face_tag > 0, unpaired, err_msg=f)
        if lines:
            assert len(lines) == int(unpaired.sum()), f
            assert set(np.unique(m.face_tag[unpaired])) <= set(lines), f
        else:
            assert (m.face_tag[unpaired] == 1).all(), f
    # the isentropic-vortex example runs through the oracle with its one boundary condition
    m = read_gmsh(os.path.join(REF_EXAMPLES, "euler", "isentropicVortex", "grid.msh"))
    o = oracle_lib.Oracle(m, 3, oracle_lib.EQ_EULER, (1.4, 0.0, 0.0),
                          bcs=((oracle_lib.BC_VORTEX, (1.0, 0.0, 5.0, 0.0, 1.4, 5.0)),))
    x, y = o.node_coords()
    from apollo_b200 import problems
    U = np.ascontiguousarray(problems.vortex_ic(x, y, 5, x0=5.0, y0=0.0, beta=5.0))
    rhs, sugg = o.rhs(U)
    assert o.error == 0 and np.isfinite(rhs).all() and sugg > 0
