"""EnSight Gold output of the host layer (EnsightSeries in cfdv_b200/host/cfdv_host.hpp; the
reference's EnsightOut.h:9-13 is an empty stub, so there is nothing to compare against): the
files are read back by a small parser of the EnSight Gold ASCII format and checked against
the mesh and against NodeUnpack of U (the same primitives the Tecplot writer prints)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import get_case
from test_tecplot_output import emit  # noqa: F401  (fixture: builds tests/emu/tecplot_emit)


def _read_geo(path):
    with open(path) as f:
        lines = [ln.rstrip("\n") for ln in f]
    assert lines[2] == "node id off" and lines[3] == "element id off"
    assert lines[4] == "part" and int(lines[5]) == 1 and lines[7] == "coordinates"
    nn = int(lines[8])
    xyz = np.array([float(v) for v in lines[9:9 + 3 * nn]]).reshape(3, nn).T
    k = 9 + 3 * nn
    etype, ne = lines[k], int(lines[k + 1])
    conn = np.array([[int(v) for v in ln.split()] for ln in lines[k + 2:k + 2 + ne]])
    assert len(lines) == k + 2 + ne
    return xyz, etype, conn


def _read_var(path, header):
    with open(path) as f:
        lines = [ln.rstrip("\n") for ln in f]
    assert lines[1] == "part" and int(lines[2]) == 1 and lines[3] == header
    return np.array([float(v) for v in lines[4:]])


def _read_case(path):
    with open(path) as f:
        text = f.read()
    head, time = text.split("\nTIME\n")
    assert head.startswith("FORMAT\ntype: ensight gold\n")
    assert "model: cfdv.geo" in head
    variables = [ln for ln in head.split("VARIABLE\n")[1].splitlines() if ln.strip()]
    tl = time.splitlines()
    nsteps = int(tl[1].split(":")[1])
    times = [float(v) for v in tl[tl.index("time values:") + 1:]]
    assert len(times) == nsteps
    return variables, times


@pytest.mark.parametrize("name", ["lid8", "plate20", "ramp4", "cyl4"])
def test_ensight_series(emit, oracle_lib, name):
    from cfdv_b200 import meshgen as mg
    case = get_case(name)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    s = o.fdvparam(U)
    nd, nn, ne = case.ndim, case.n_nodes, case.n_elements
    with tempfile.TemporaryDirectory() as d:
        cdir = os.path.join(d, "case")
        mg.write_case(case, cdir)
        U.tofile(os.path.join(d, "U.bin"))
        s.tofile(os.path.join(d, "s.bin"))
        out = os.path.join(d, "ens")
        subprocess.run([emit, cdir, os.path.join(d, "U.bin"), os.path.join(d, "s.bin"), "0", "0.25", out, "ensight"],
                       check=True)
        variables, times = _read_case(os.path.join(out, "cfdv.case"))
        xyz, etype, conn = _read_geo(os.path.join(out, "cfdv.geo"))
        fields = {}
        for step in range(2):
            for var in ("rho", "T", "p", "velocity"):
                fields[(var, step)] = _read_var(os.path.join(out, f"cfdv.{var}.{step:05d}"), "coordinates")
            for k in range(1, 5):
                fields[(f"s{k}", step)] = _read_var(os.path.join(out, f"cfdv.s{k}.{step:05d}"), etype)
    assert times == [0.25, 0.5]
    assert len(variables) == 8
    assert variables[1] == "vector per node: 1 velocity cfdv.velocity.*****"
    assert etype == ("quad4" if nd == 2 else "hexa8")
    x = case.nodes[:, :nd]
    np.testing.assert_allclose(xyz[:, :nd], x, rtol=1e-5, atol=1e-12)  # %12.5e
    if nd == 2:
        assert np.all(xyz[:, 2] == 0.0)
    assert np.array_equal(conn, case.elements[:, : 4 if nd == 2 else 8] + 1)
    # NodeUnpack of U (NodeUnpack.h:9-29)
    Ur = U.reshape(nn, nd + 2)
    rho = Ur[:, 0]
    v = Ur[:, 1:nd + 1] / rho[:, None]
    e = Ur[:, nd + 1] / rho - 0.5 * np.sum(v * v, axis=1)
    gamma, M = float(case.aero["gamma"]), float(case.aero["M"])
    Cv = 1.0 / gamma / (gamma - 1.0) / (M * M)
    for step in range(2):
        np.testing.assert_allclose(fields[("rho", step)], rho, rtol=1e-5)
        np.testing.assert_allclose(fields[("T", step)], e / Cv, rtol=1e-5, atol=1e-300)
        np.testing.assert_allclose(fields[("p", step)], rho * (gamma - 1.0) * e, rtol=1e-5, atol=1e-300)
        vel = fields[("velocity", step)].reshape(3, nn).T
        np.testing.assert_allclose(vel[:, :nd], v, rtol=1e-5, atol=1e-5 * np.abs(v).max() + 1e-300)
        assert np.all(vel[:, nd:] == 0.0)
        for k in range(4):
            np.testing.assert_allclose(fields[(f"s{k + 1}", step)], s.reshape(ne, 4)[:, k], rtol=1e-5, atol=1e-300)
