"""The oracle restatement against the reference build on the full-size flat plate.

tests/golden/plate200x100.npz holds 25 steps of the CFDV reference sources, compiled
unmodified, on the 200x100 plate (M 3, Re 1e4, CFL 1, the reference's GMRES(30) with one
restart).  The restatement (oracle/cfdv_oracle.cpp) must reproduce them bit for bit: dt,
every Givens estimate, g(m), the RMS line and U -- the same bar as on the small cases, at
the size the headline benchmark runs."""
import os

import numpy as np

from conftest import GOLDEN

from cfdv_b200 import meshgen as mg


def test_oracle_reproduces_reference_plate_25_steps_bitwise(oracle_lib):
    case = mg.FULL["plate"]()
    g = dict(np.load(os.path.join(GOLDEN, "plate200x100.npz")))
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    cl = o.cleng()
    dofs = g["dof_sample"]
    for k in range(int(g["steps"])):
        U, _, dt, rms, rep = o.step(U, float(case.control["cfl"]), int(case.control["gmresiter"]),
                                    int(case.control["gmresrestart"]), mode=0, cleng=cl)
        assert dt == g[f"dt@{k}"][0]
        assert np.array_equal(rep["est"], g[f"est@{k}"])
        assert np.array_equal(rep["gfinal"], g[f"gfinal@{k}"])
        assert np.array_equal(U[dofs], g[f"Usample@{k}"])
        assert np.array_equal(rms, g[f"rms@{k}"])
    assert np.array_equal(U, g[f"U@{int(g['steps']) - 1}"])
