"""VTK frame output (apollo_b200.vtk): what is written reads back unchanged."""
import os

import numpy as np

from apollo_b200.mesh import jittered_square
from apollo_b200.vtk import read_vtu, write_frame, write_vtu


def test_vtu_round_trip(tmp_path):
    m = jittered_square(6, (0.0, 0.0), (2.0, 1.0), seed=1, periodic=False)
    U = np.random.default_rng(0).standard_normal((m.K, 10, 4))
    w = np.full(10, 0.1)
    path = str(tmp_path / "f.vtu")
    write_vtu(path, m, U, averages=w, time=0.25)
    a = read_vtu(path)
    np.testing.assert_array_equal(a["Points"][:, 0], m.vx)
    np.testing.assert_array_equal(a["Points"][:, 1], m.vy)
    np.testing.assert_array_equal(a["connectivity"].reshape(-1, 3), m.etov)
    np.testing.assert_array_equal(a["offsets"], 3 * np.arange(1, m.K + 1))
    assert (a["types"] == 5).all()
    np.testing.assert_array_equal(a["solution"], U.reshape(m.K, -1))
    np.testing.assert_allclose(a["rho"], U[..., 0].mean(axis=1), rtol=1e-14)
    assert a["TIME"][0] == 0.25


def test_frame_name_follows_apollo(tmp_path):
    m = jittered_square(4, periodic=False)
    p = write_frame("vortex", 7, m, np.zeros((m.K, 6, 1)), directory=str(tmp_path))
    assert os.path.basename(p) == "vortex_7.vtu" and os.path.exists(p)
