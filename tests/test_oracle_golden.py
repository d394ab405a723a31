"""The CPU restatement (oracle/cfdv_oracle.cpp) against golden outputs of the reference
itself (tests/golden/*.npz, written by tests/golden/make_golden.py from oracle/_ref)."""
import numpy as np
import pytest

from conftest import ADAPTIVE_CASES, SMALL_CASES, get_case, golden, rel_err, elem_rel_err
from golden.make_golden import case_digest


@pytest.mark.parametrize("name", SMALL_CASES + ADAPTIVE_CASES)
def test_case_inputs_match_fixture(name):
    assert str(golden(name)["digest"]) == case_digest(get_case(name))


@pytest.mark.parametrize("name", SMALL_CASES + ADAPTIVE_CASES)
def test_setup_matches_reference(name, oracle_lib):
    g, case = golden(name), get_case(name)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    assert rel_err(U, g["U_init"]) == 0.0
    assert rel_err(o.cleng(), g["cleng"]) == 0.0
    assert (o.dirichlet() == g["dirichlet"]).all()
    assert rel_err(o.fdvparam(U).ravel(), g["s1234"]) == 0.0
    assert o.cfl(U, float(case.control["cfl"])) == g["dt@0"][0]


@pytest.mark.parametrize("name", SMALL_CASES + ADAPTIVE_CASES)
def test_formation_matches_reference(name, oracle_lib):
    g, case = golden(name), get_case(name)
    o = oracle_lib.Oracle(case)
    R, rhs = o.form(o.init_U(), g["dt_dump"][0], apply_bc=True)
    el = g["elements"]
    # same arithmetic order as the reference: agreement to the last bit
    assert elem_rel_err(R[el], g["R_bc"]) <= 1e-15
    assert rel_err(rhs[el], g["rhs_bc"]) <= 1e-15


@pytest.mark.parametrize("name", SMALL_CASES + ADAPTIVE_CASES)
def test_reference_steps_match(name, oracle_lib):
    g, case = golden(name), get_case(name)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    cl = o.cleng()
    m, r, cfl = int(case.control["gmresiter"]), int(case.control["gmresrestart"]), float(case.control["cfl"])
    for s in range(int(g["steps"])):
        U, U0, dt, rms, rep = o.step(U, cfl, m, r, mode=0, cleng=cl)
        assert dt == g[f"dt@{s}"][0]
        assert rep["tol"] == pytest.approx(g[f"tol@{s}"][0], rel=1e-15)
        assert len(rep["est"]) == len(g[f"est@{s}"])
        assert rel_err(rep["est"], g[f"est@{s}"]) <= 1e-12
        assert rel_err(rep["gfinal"], g[f"gfinal@{s}"]) <= 1e-12
        assert rel_err(U, g[f"U@{s}"]) <= 1e-14
        assert rel_err(rms, g[f"rms@{s}"]) <= 1e-12


def test_correct_gmres_reaches_tolerance(oracle_lib):
    case = get_case("lid8")
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    dt = o.cfl(U, 0.5)
    R, rhs = o.form(U, dt)
    du, rep = o.gmres_correct(R, rhs, 20, 50, 1e-10)
    assert rep["true_rel_res"] < 1e-10
    # the reference solver's own back substitution leaves a much larger residual
    _, rep_ref = o.gmres_ref(R, rhs, 20, 1)
    assert rep_ref["true_rel_res"] > 1e-4


def test_transposed_product_is_adjoint(oracle_lib):
    case = get_case("ramp4")
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    R, _ = o.form(U, o.cfl(U, 0.25))
    rng = np.random.default_rng(3)
    x, y = rng.standard_normal(o.n_dof), rng.standard_normal(o.n_dof)
    lhs = y @ o.matvec(R, x)
    rhs = x @ o.matvec(R, y, transpose=True)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
