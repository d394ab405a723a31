"""The ASCII -> binary case converter (cfdv_b200/cfdv_convert: cfdv_host::convert_ascii, the
reference's CONVERT tool, ConvertMain.cpp / AsciiLoad.h): a case written in the reference's
ASCII form with the conserved state from LoadBinary's conversion converts back to the same
binary case (mesh and codes exactly, primitives to the rounding of NodeUnpack), and the
reference build reads the converted directory back to the same state."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, get_case, rel_err

CONVERT = os.path.join(ROOT, "cfdv_b200", "cfdv_convert")
REF = os.path.join(ROOT, "oracle", "_ref", "cfdv_ref")


@pytest.fixture(scope="module")
def convert():
    src = [os.path.join(ROOT, "cfdv_b200", "host", f) for f in ("cfdv_convert.cpp", "cfdv_host.hpp")]
    if not os.path.exists(CONVERT) or os.path.getmtime(CONVERT) < max(os.path.getmtime(f) for f in src):
        subprocess.run(["make", "-C", os.path.join(ROOT, "cfdv_b200"), "cfdv_convert"], check=True,
                       capture_output=True)
    return CONVERT


@pytest.mark.parametrize("name", ["lid8", "plate20", "ramp4", "cyl4", "lid8_adap", "ramp4_adap"])
def test_ascii_case_converts_to_the_binary_case(convert, oracle_lib, name):
    from cfdv_b200 import meshgen as mg
    case = get_case(name)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    with tempfile.TemporaryDirectory() as d:
        a, b = os.path.join(d, "ascii"), os.path.join(d, "bin")
        mg.write_ascii_case(case, a, U)
        subprocess.run([convert, a, b], check=True, capture_output=True)
        back = mg.read_case(b)
        ref = None
        if os.path.exists(REF):
            ref = oracle_lib.run_reference(b, os.path.join(d, "r.rec"), steps=1)
    nd = case.ndim
    assert np.array_equal(back.elements, case.elements)
    assert np.array_equal(back.nodes[:, : nd + 1], case.nodes[:, : nd + 1])  # x, rho
    np.testing.assert_allclose(back.nodes[:, nd + 1:], case.nodes[:, nd + 1:], rtol=1e-14, atol=1e-15)
    assert {k: str(v) for k, v in back.control.items()} == {k: str(v) for k, v in case.control.items()}
    if case.adap_elements is not None:
        assert np.array_equal(back.adap_elements, case.adap_elements)
        assert np.array_equal(back.adap_hnm, case.adap_hnm)
    if ref is not None:
        assert rel_err(ref["U_init"], U) <= 1e-14


def test_missing_node_is_an_error(convert, oracle_lib):
    from cfdv_b200 import meshgen as mg
    case = get_case("lid8")
    U = oracle_lib.Oracle(case).init_U()
    with tempfile.TemporaryDirectory() as d:
        a = os.path.join(d, "ascii")
        mg.write_ascii_case(case, a, U)
        lines = open(os.path.join(a, "nodes")).read().splitlines()
        open(os.path.join(a, "nodes"), "w").write("\n".join(lines[:-1]) + "\n")
        r = subprocess.run([convert, a, os.path.join(d, "bin")], capture_output=True, text=True)
    assert r.returncode == 1 and "is not defined" in r.stderr
