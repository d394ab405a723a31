"""Pin the restatement against the reference build run live (oracle/_ref/cfdv_ref),
on longer runs than the fixtures hold.  Skipped where the reference build is absent."""
import os
import tempfile

import pytest

from conftest import get_case, rel_err
from cfdv_b200 import meshgen as mg

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "cfdv_ref")
pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="reference build oracle/_ref not present")


@pytest.mark.parametrize("name,steps", [("lid32", 5), ("plate20", 10)])
def test_restatement_tracks_reference(name, steps, oracle_lib):
    case = mg.SMALL[name]() if name in mg.SMALL else get_case(name)
    with tempfile.TemporaryDirectory() as d:
        mg.write_case(case, d)
        rec = oracle_lib.run_reference(d, os.path.join(d, "o.rec"), steps=steps)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    cl = o.cleng()
    for s in range(steps):
        U, _, dt, rms, rep = o.step(U, float(case.control["cfl"]), int(case.control["gmresiter"]),
                                    int(case.control["gmresrestart"]), cleng=cl)
        assert dt == rec[f"dt@{s}"][0]
        assert rel_err(rep["est"], rec[f"est@{s}"]) <= 1e-12
    assert rel_err(U, rec[f"U@{steps - 1}"]) <= 1e-13
