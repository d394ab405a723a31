"""Synthetic cases: reference binary format round trip and the configured sizes."""
import os
import tempfile

import numpy as np

from cfdv_b200 import meshgen as mg


def test_round_trip():
    c = mg.lid(8)
    with tempfile.TemporaryDirectory() as d:
        mg.write_case(c, d)
        assert os.path.getsize(os.path.join(d, "binarynodes")) == c.n_nodes * 6 * 8
        assert os.path.getsize(os.path.join(d, "binaryelements")) == c.n_elements * 8 * 4
        r = mg.read_case(d)
    assert np.array_equal(r.nodes, c.nodes) and np.array_equal(r.elements, c.elements)
    assert int(r.control["gmresiter"]) == 20 and float(r.aero["M"]) == 0.1


def test_sizes_of_configured_workloads():
    assert (mg.lid(32).n_elements, mg.lid(32).n_nodes) == (1024, 1089)
    p = mg.plate(200, 100)
    assert (p.n_elements, p.n_nodes) == (20000, 20301)
    r = mg.ramp(128, 64, 32)
    assert (r.n_elements, r.n_nodes) == (262144, 276705)
    cyl = mg.cylinder()
    wall = np.isclose(np.hypot(cyl.nodes[:, 0], cyl.nodes[:, 1]), 0.5)
    assert wall.sum() == 2048


def test_positive_jacobians():
    for c in (mg.ramp(8, 4, 4), mg.cylinder(6, 8, 4), mg.duct(8, 4, 4)):
        x = c.nodes[:, :3][c.conn]
        # hex volume sign from the (0,1),(0,3),(0,4) edge triple
        v = np.einsum("ij,ij->i", x[:, 1] - x[:, 0], np.cross(x[:, 3] - x[:, 0], x[:, 4] - x[:, 0]))
        assert (v > 0).all()
