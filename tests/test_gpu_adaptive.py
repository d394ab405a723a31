"""Adaptive (hanging-node) elements on the device (cfdv_set_adaptive; the reference's adap
file, LoadBinary.h:247-261, and the Hnm transforms of MeshRefine2D.h:877-952): argument
checks, the identity Hnm, steps of the textbook solve against the oracle, and the discrete
adjoint against the tangent-linear run on an adaptive mesh.  Formation and the reference
GMRES history against the reference's own outputs are in test_gpu_parity.py."""
import numpy as np
import pytest

from conftest import get_case, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from cfdv_b200 import gpu as G
    return G


def _solver(G, case):
    s = G.FDVSolver(case)
    s.load_node_records()
    return s


def test_set_adaptive_rejects_bad_input(gpu):
    case = get_case("lid8")
    H = np.eye(4)[None]
    with _solver(gpu, case) as s:
        for els, h in (([case.n_elements], H), ([-1], H), ([3, 3], np.concatenate([H, H])),
                       ([3], H * np.nan)):
            with pytest.raises(gpu.CfdvError) as e:
                s.set_adaptive(els, h)
            assert e.value.code == 1  # CFDV_ERR_ARG
        s.set_adaptive([], np.zeros((0, 4, 4)))  # clearing is allowed


@pytest.mark.parametrize("name", ["lid8", "ramp4"])
def test_identity_hnm_reproduces_plain_elements(gpu, name):
    """Hnm = I multiplies by one and adds zeros: the element matrices are bit for bit the
    plain ones, boundary faces included."""
    case = get_case(name)
    nn = case.nnod
    with _solver(gpu, case) as s:
        dt = s.cfl(float(case.control["cfl"]))
        s.form(dt)
        R0, r0 = s.element_matrices()
        s.set_adaptive(np.arange(case.n_elements), np.broadcast_to(np.eye(nn), (case.n_elements, nn, nn)))
        s.form(dt)
        R1, r1 = s.element_matrices()
    assert np.array_equal(R0, R1) and np.array_equal(r0, r1)


@pytest.mark.parametrize("name", ["lid8_adap", "ramp4_adap"])
def test_textbook_steps_match_oracle(gpu, oracle_lib, name):
    """Three textbook steps (GMRES to 1e-12) on the adaptive mesh against the oracle."""
    case = get_case(name)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    cl = o.cleng()
    cfl = float(case.control["cfl"])
    with _solver(gpu, case) as s:
        for _ in range(3):
            U = o.step(U, cfl, 30, 50, mode=1, rtol=1e-12, cleng=cl)[0]
            s.step(cfl, mode=gpu.GMRES_CORRECT, m=30, restarts=50, rtol=1e-12)
        Ug = s.get_state()
    assert rel_err(Ug, U) <= 1e-8


def test_adjoint_matches_tangent_on_adaptive_mesh(gpu):
    """Mach and wall-temperature gradients of the wall-force functional on the cylinder with
    adaptive elements (some on the wall): reverse sweep against the tangent-linear run."""
    case = get_case("cyl4_adap")
    assert np.isin(case.adap_elements, np.where((case.bc == 1).any(axis=1))[0]).any()
    with _solver(gpu, case) as s:
        r = s.adjoint(4, 0.5, checkpoint_every=2, m=40, rtol=1e-12)
        J, dJm = s.tangent(4, 0.5, dmach=1.0, m=40, rtol=1e-12)
        v = np.random.default_rng(5).standard_normal(len(r["wall_nodes"]))
        _, dJt = s.tangent(4, 0.5, dT_wall=v, m=40, rtol=1e-12)
    assert J == pytest.approx(r["J"], rel=1e-12)
    assert r["dJ_dmach"] == pytest.approx(dJm, rel=1e-8)
    assert float(r["dJ_dtnode"] @ v) == pytest.approx(dJt, rel=1e-8)
