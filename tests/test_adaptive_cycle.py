"""The refinement cycle of the reference: mark, refine on the host, re-upload, step.

The reference refines at startup when asked (main.cpp:139-148): NodeUnpack, NodeCheck,
AdaptiveRefineList -- the elements whose FDVParam s1 exceeds 0.8 (RefineListAdaptive.h:25-36)
plus their dependencies -- and MeshRefine2D, then Save; the next run loads the refined case
with its "adap" file.  The refinement stays on the host, in the reference's own code
(oracle/_ref/cfdv_ref --refine runs it on the state after some steps and records the marks
and the refined case).  These tests check the pieces around it:

  CPU  the oracle steps the refined case exactly as the reference does (bitwise), so the
       refined-case round trip (records -> case directory -> both loaders) is sound;
  GPU  one context steps the original case, its device marks (cfdv_refine_marks) equal the
       reference's s1 > 0.8 list, then the refined case goes into the SAME context
       (cfdv_upload_mesh, the node records, cfdv_set_adaptive) and its steps match the
       reference stepping the refined case: the Givens history and U to <= 1e-10."""
import os
import tempfile

import numpy as np
import pytest

from conftest import ROOT, get_case, rel_err

from cfdv_b200 import meshgen as mg

REF = os.path.join(ROOT, "oracle", "_ref", "cfdv_ref")
# (case, steps before refining, steps after).  2D only: on the hex8 ramp the reference's refined
# case gives NaN in its own first solve (its 3D refinement path), so it is no parity target.
CASES = [("lid8", 2, 3), ("plate20", 2, 3), ("plate20", 5, 3)]
needs_ref = pytest.mark.skipif(not os.path.exists(REF), reason="reference build (oracle/_ref) not present")


def refined_case(base, rec):
    """The case the reference's Save would write after MeshRefine2D (records of --refine)."""
    nd, nnod, nface = base.ndim, base.nnod, base.nface
    nodes = rec["refined_nodes"].reshape(-1, 2 * nd + 2)
    conn = rec["refined_conn"].reshape(-1, nnod)
    bc = rec["refined_bc"].reshape(-1, nface)
    assert np.array_equal(rec["refined_node_numbers"], np.arange(len(nodes)))
    control = dict(base.control)
    control["nodes"], control["elements"] = len(nodes), len(conn)
    c = mg.Case(base.name + "_refined", nd, nodes, np.concatenate([conn, bc], axis=1).astype(np.int32), control,
                dict(base.aero))
    adap = rec["refined_adap"]
    if len(adap):
        # Hnm(N, M) recorded at N + nnod*M
        hnm = np.transpose(rec["refined_hnm"].reshape(len(adap), nnod, nnod), (0, 2, 1))
        c = mg.with_adaptive(c, adap, hnm, rec["refined_levels"])
    return c


def reference_cycle(name, before, after):
    """(original case, records of the refining run, refined case, records of the refined run)"""
    from oracle import oracle as O
    case = get_case(name)
    with tempfile.TemporaryDirectory() as d:
        a, b = os.path.join(d, "a"), os.path.join(d, "b")
        mg.write_case(case, a)
        rec = O.run_reference(a, os.path.join(d, "a.rec"), steps=before, extra=["--refine"])
        ref_case = refined_case(case, rec)
        mg.write_case(ref_case, b)
        rec2 = O.run_reference(b, os.path.join(d, "b.rec"), steps=after)
    return case, rec, ref_case, rec2


@needs_ref
@pytest.mark.parametrize("name,before,after", CASES)
def test_oracle_steps_refined_case_like_reference(oracle_lib, name, before, after):
    case, rec, ref_case, rec2 = reference_cycle(name, before, after)
    assert len(rec["refine_marks"]) > 0 and ref_case.n_elements > case.n_elements
    o = oracle_lib.Oracle(ref_case)
    U = o.init_U()
    assert np.array_equal(U, rec2["U_init"])
    cl = o.cleng()
    m, r, cfl = int(case.control["gmresiter"]), int(case.control["gmresrestart"]), float(case.control["cfl"])
    for k in range(after):
        U, _, dt, _, rep = o.step(U, cfl, m, r, mode=0, cleng=cl)
        assert dt == rec2[f"dt@{k}"][0]
        assert np.array_equal(rep["est"], rec2[f"est@{k}"])
        assert np.array_equal(U, rec2[f"U@{k}"])


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("name,before,after", CASES)
def test_gpu_refine_reupload_cycle_matches_reference(name, before, after):
    from cfdv_b200 import gpu as G
    case, rec, ref_case, rec2 = reference_cycle(name, before, after)
    m, r, cfl = int(case.control["gmresiter"]), int(case.control["gmresrestart"]), float(case.control["cfl"])
    with G.FDVSolver(case) as s:
        s.load_node_records()
        for _ in range(before):
            s.step(cfl, mode=G.GMRES_REFERENCE, m=m, restarts=r)
        marks = s.refine_marks(0.8)
        assert np.array_equal(marks, rec["refine_marks"])
        # the host refined the mesh (the reference's MeshRefine2D); hand it back to the same context
        s.upload_case(ref_case)
        s.load_node_records()
        assert rel_err(s.get_state(), rec2["U_init"]) == 0.0
        for k in range(after):
            rep = s.step(cfl, mode=G.GMRES_REFERENCE, m=m, restarts=r)
            assert rep["dt"] == pytest.approx(rec2[f"dt@{k}"][0], rel=1e-12)
            assert len(rep["est"]) == len(rec2[f"est@{k}"])
            assert rel_err(rep["est"], rec2[f"est@{k}"]) <= 1e-10
            assert rel_err(s.get_state(), rec2[f"U@{k}"]) <= 1e-10
