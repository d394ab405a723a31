"""Checkpoints of the host layer (save_case in cfdv_b200/host/cfdv_host.hpp, the reference's
Save: MPIBinaryConfiguration.h:148-161, SaveBinary.h): the saved case directory holds the
state as binary node records that LoadBinary reads (2D and 3D), with control iter set, and a
run resumed from it continues the uninterrupted run."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, get_case
from test_tecplot_output import emit  # noqa: F401  (fixture: builds tests/emu/tecplot_emit)


def _save(emit, case, U, iter_, d):
    from cfdv_b200 import meshgen as mg
    cdir = os.path.join(d, "case")
    mg.write_case(case, cdir)
    U.tofile(os.path.join(d, "U.bin"))
    np.zeros(case.n_elements * 4).tofile(os.path.join(d, "s.bin"))
    out = os.path.join(d, "ckpt")
    subprocess.run([emit, cdir, os.path.join(d, "U.bin"), os.path.join(d, "s.bin"), str(iter_), "0", out, "save"],
                   check=True)
    return os.path.join(out, str(iter_))


@pytest.mark.parametrize("name", ["lid8", "plate20", "ramp4", "cyl4"])
def test_saved_records_round_trip(emit, oracle_lib, name):
    """Saving the initial state reproduces the case's own records (NodeUnpack of U built by
    LoadBinary): coordinates and density exactly, velocity and temperature to rounding."""
    from cfdv_b200 import meshgen as mg
    case = get_case(name)
    U = oracle_lib.Oracle(case).init_U()
    with tempfile.TemporaryDirectory() as d:
        sdir = _save(emit, case, U, 0, d)
        back = mg.read_case(sdir)
    nd = case.ndim
    assert back.nodes.shape == case.nodes.shape and back.elements.shape == case.elements.shape
    assert np.array_equal(back.elements, case.elements)
    assert np.array_equal(back.nodes[:, : nd + 1], case.nodes[:, : nd + 1])  # x, rho
    np.testing.assert_allclose(back.nodes[:, nd + 1:], case.nodes[:, nd + 1:], rtol=1e-14, atol=1e-15)
    assert int(back.control["iter"]) == 0
    assert set(back.aero) == set(case.aero)
    for k, v in case.aero.items():
        assert float(back.aero[k]) == float(v)


@pytest.mark.parametrize("name", ["lid8", "ramp4"])
def test_resumed_run_continues(emit, oracle_lib, name):
    """Two oracle steps, a checkpoint, one step from the reloaded checkpoint: the same state as
    three uninterrupted steps (textbook solve to 1e-12), to the rounding of the record round
    trip.  The reference build reads the saved directory as a case."""
    from cfdv_b200 import meshgen as mg
    case = get_case(name)
    o = oracle_lib.Oracle(case)
    cfl = float(case.control["cfl"])
    U = o.init_U()
    cl = o.cleng()
    for _ in range(2):
        U = o.step(U, cfl, 30, 50, mode=1, rtol=1e-12, cleng=cl)[0]
    U3 = o.step(U, cfl, 30, 50, mode=1, rtol=1e-12, cleng=cl)[0]
    with tempfile.TemporaryDirectory() as d:
        sdir = _save(emit, case, U, 2, d)
        back = mg.read_case(sdir)
        ref_bin = os.path.join(ROOT, "oracle", "_ref", "cfdv_ref")
        if os.path.exists(ref_bin):
            rec = oracle_lib.run_reference(sdir, os.path.join(d, "r.rec"), steps=1)
            assert len(rec) > 0
    o2 = oracle_lib.Oracle(back)
    Ur = o2.init_U()
    assert np.abs(Ur - U).max() <= 1e-13 * np.abs(U).max()
    Ur3 = o2.step(Ur, cfl, 30, 50, mode=1, rtol=1e-12, cleng=o2.cleng())[0]
    assert np.abs(Ur3 - U3).max() <= 1e-10 * np.abs(U3).max()
