"""Edge cases of the persistent GMRES solve (engine 0): Krylov dimensions at and beyond the
delayed-CGS2 limit (m + 2 <= 64 partial slots; larger m runs MGS in the same kernel), a zero
right-hand side (||b|| = 0 computed inside the kernel: du = 0, nothing iterated), and zero
restarts (only the final residual)."""
import numpy as np
import pytest

from conftest import get_case, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from cfdv_b200 import gpu as G
    return G


def _formed(G, name):
    case = get_case(name)
    s = G.FDVSolver(case)
    s.load_node_records()
    dt = s.cfl(float(case.control["cfl"]))
    s.form(dt, precision=G.PREC_MIXED)
    return s


@pytest.mark.parametrize("name", ["lid8", "ramp4"])
@pytest.mark.parametrize("m", [62, 70])
def test_large_krylov_dimension(gpu, oracle_lib, name, m):
    """m = 62 is the largest delayed-CGS2 basis; m = 70 falls back to MGS.  Both reach the
    tolerance and agree with the host-driven MGS solve."""
    with _formed(gpu, name) as s:
        r0 = s.gmres(mode=gpu.GMRES_CORRECT, m=m, restarts=20, rtol=1e-10, engine=0, orth=2)
        d0 = s.du()
        r1 = s.gmres(mode=gpu.GMRES_CORRECT, m=m, restarts=20, rtol=1e-10, engine=1)
        d1 = s.du()
    assert r0["true_rel_res"] < 1e-10 and r1["true_rel_res"] < 1e-10
    assert rel_err(d0, d1) <= 1e-7


def test_zero_rhs_gives_zero_update(gpu):
    case = get_case("lid8")
    Ke = case.nnod * case.neqn
    rng = np.random.default_rng(1)
    R = np.eye(Ke)[None] + 0.01 * rng.standard_normal((case.n_elements, Ke, Ke))
    with gpu.FDVSolver(case) as s:
        s.load_node_records()
        s.set_element_matrices(np.ascontiguousarray(R), np.zeros((case.n_elements, Ke)))
        rep = s.gmres(mode=gpu.GMRES_CORRECT, m=20, restarts=5, rtol=1e-8, engine=0)
        du = s.du()
    assert rep["bnorm"] == 0.0 and rep["true_rel_res"] == 0.0
    assert rep["matvecs"] == 0 and not du.any()


def test_zero_restarts_reports_the_initial_residual(gpu):
    with _formed(gpu, "lid8") as s:
        rep = s.gmres(mode=gpu.GMRES_CORRECT, m=20, restarts=0, rtol=1e-8, engine=0)
        du = s.du()
    assert not du.any()
    assert rep["true_rel_res"] == pytest.approx(1.0, rel=1e-12)  # r = b - A 0
