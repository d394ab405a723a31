"""Adaptive (hanging-node) cases on the CPU: the reference's "adap" file (LoadBinary.h:247-261,
TensorStream.h:95-145) written and read back by cfdv_b200.meshgen, the identity Hnm in the
oracle, and, where the reference build is present, the oracle against the reference run on
an adaptive case directly (the committed fixtures tests/golden/*_adap.npz hold the same
comparison for runs without it; test_oracle_golden.py)."""
import os
import tempfile

import numpy as np
import pytest

from conftest import ROOT, get_case, rel_err, elem_rel_err

REF = os.path.join(ROOT, "oracle", "_ref", "cfdv_ref")


@pytest.mark.parametrize("name", ["lid8_adap", "ramp4_adap"])
def test_adap_file_round_trip(name):
    from cfdv_b200 import meshgen as mg
    case = get_case(name)
    with tempfile.TemporaryDirectory() as d:
        mg.write_case(case, d)
        with open(os.path.join(d, "adap")) as f:
            first = f.readline().split()
        back = mg.read_case(d)
    nn = case.nnod
    # elno adap refine_level, then the Tensor: type, ndim, extents, data in index order N + nnod*M
    assert first[:7] == [str(case.adap_elements[0]), "1", "1", "double", "2", str(nn), str(nn)]
    assert np.array_equal(np.array(first[7:], float), case.adap_hnm[0].T.ravel())
    assert np.array_equal(back.adap_elements, case.adap_elements)
    assert np.array_equal(back.adap_hnm, case.adap_hnm)
    assert int(back.control["adap"]) == 1


@pytest.mark.parametrize("name", ["lid8", "ramp4"])
def test_identity_hnm_is_the_plain_element(oracle_lib, name):
    from cfdv_b200 import meshgen as mg
    case = get_case(name)
    ident = mg.with_adaptive(case, np.arange(case.n_elements),
                             np.broadcast_to(np.eye(case.nnod), (case.n_elements, case.nnod, case.nnod)))
    o, oi = oracle_lib.Oracle(case), oracle_lib.Oracle(ident)
    U = o.init_U()
    dt = o.cfl(U, float(case.control["cfl"]))
    R, r = o.form(U, dt)
    Ri, ri = oi.form(U, dt)
    assert np.array_equal(R, Ri) and np.array_equal(r, ri)


@pytest.mark.skipif(not os.path.exists(REF), reason="reference build oracle/_ref not present")
@pytest.mark.parametrize("name", ["lid8_adap", "ramp4_adap"])
def test_oracle_matches_reference_run(oracle_lib, name):
    from cfdv_b200 import meshgen as mg
    case = get_case(name)
    with tempfile.TemporaryDirectory() as d:
        mg.write_case(case, d)
        rec = oracle_lib.run_reference(d, os.path.join(d, "out.rec"), steps=2, dump_step=0)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    Ke = case.nnod * case.neqn
    R, rhs = o.form(U, float(rec["dt_dump"][0]))
    assert elem_rel_err(R, rec["R_bc"].reshape(case.n_elements, Ke, Ke)) <= 1e-15
    assert rel_err(rhs, rec["rhs_bc"].reshape(case.n_elements, Ke)) <= 1e-15
    cl = o.cleng()
    m, r, cfl = int(case.control["gmresiter"]), int(case.control["gmresrestart"]), float(case.control["cfl"])
    for s in range(2):
        U = o.step(U, cfl, m, r, mode=0, cleng=cl)[0]
        assert rel_err(U, rec[f"U@{s}"]) <= 1e-14
