"""Edge cases of the persistent GMRES solve (engine 0): Krylov dimensions at and beyond the
delayed-CGS2 limit (m + 2 <= 64 partial slots; larger m runs MGS in the same kernel), a zero
right-hand side (||b|| = 0 computed inside the kernel: du = 0, nothing iterated), zero
restarts (only the final residual), and the 2D neighbour syncs of the delayed-CGS2 step
against grid barriers."""
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


@pytest.mark.parametrize("name", ["lid8", "lid32", "plate20", "lid8_adap", "plate200x100"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("precond", [True, False])
def test_neighbour_syncs_match_grid_barriers(gpu, name, prec, precond):
    """orth 2 replaces two of the three grid barriers of a 2D delayed-CGS2 step by waits on the
    blocks owning neighbouring nodes and elements; orth 3 keeps grid barriers.  The arithmetic
    and its order are the same, so the solves agree bit for bit, and repeated runs with the
    neighbour syncs do too.  lid8 has fewer elements than blocks (empty blocks and sets)."""
    if name == "plate200x100":
        from cfdv_b200 import meshgen as mg
        case = mg.plate(200, 100)
    else:
        case = get_case(name)
    p = gpu.PREC_MIXED if prec == "mixed" else gpu.PREC_FP64
    runs = []
    with gpu.FDVSolver(case) as s:
        s.load_node_records()
        s.form(s.cfl(float(case.control["cfl"])), precision=gpu.PREC_MIXED)
        for orth in (3, 2, 2):
            r = s.gmres(mode=gpu.GMRES_CORRECT, m=30, restarts=80, rtol=1e-8, precision=p, engine=0,
                        precond=precond, orth=orth)
            runs.append((r, s.du()))
    (r3, d3), (r2, d2), (r2b, d2b) = runs
    assert r3["true_rel_res"] < 1e-8
    for r, d in ((r2, d2), (r2b, d2b)):
        assert np.array_equal(d, d3)
        assert np.array_equal(r["est"], r3["est"])
        assert r["restarts"] == r3["restarts"] and r["true_rel_res"] == r3["true_rel_res"]


@pytest.mark.parametrize("name", ["plate20", "ramp4"])
@pytest.mark.parametrize("engine", [0, 1])
def test_step_host_equals_set_step_get(gpu, name, engine):
    """cfdv_step_host (state in and out as host arrays, one wait) gives the same state, dt and
    residual history as cfdv_set_state + cfdv_step + cfdv_get_state."""
    case = get_case(name)
    kw = dict(mode=gpu.GMRES_CORRECT, m=30, restarts=80, rtol=1e-8, precision=gpu.PREC_MIXED, engine=engine)
    with gpu.FDVSolver(case) as s:
        s.load_node_records()
        U0 = s.get_state()
        s.set_state(U0)
        r1 = s.step(float(case.control["cfl"]), **kw)
        U1 = s.get_state()
        s.set_state(np.zeros_like(U0))  # overwritten by the step's own upload
        U2 = np.empty_like(U0)
        r2 = s.step_host(float(case.control["cfl"]), U0, U2, **kw)
        U3 = s.get_state()
    assert np.array_equal(U1, U2) and np.array_equal(U2, U3)
    assert r1["dt"] == r2["dt"] and np.array_equal(r1["est"], r2["est"])


@pytest.mark.parametrize("name", ["plate20", "ramp4"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_warm_start(gpu, name, prec):
    """A solve started from the previous solution: solving the same formed system again stops
    after the one product of its initial residual, with du unchanged; and steps started from
    the previous step's dU meet the same stopping test as steps started from zero and end at
    the same state within the solver's tolerance (the first step has no previous dU)."""
    case = get_case(name)
    p = gpu.PREC_FP64 if prec == "fp64" else gpu.PREC_MIXED
    cfl = float(case.control["cfl"])
    kw = dict(mode=gpu.GMRES_CORRECT, m=30, restarts=200, rtol=1e-10, precision=p, true_residual=True)
    with gpu.FDVSolver(case) as s:
        s.load_node_records()
        s.form(s.cfl(cfl), p)
        first = s.gmres(**kw)
        du = s.du().copy()
        again = s.gmres(warm_start=True, **kw)
        assert first["matvecs"] > 1 and again["matvecs"] == 1
        assert again["true_rel_res"] < 1e-10 and np.array_equal(s.du(), du)
    runs = {}
    for warm in (False, True):
        with gpu.FDVSolver(case) as s:
            s.load_node_records()
            reps = [s.step(cfl, warm_start=warm, **kw) for _ in range(4)]
            runs[warm] = (s.get_state(), reps)
    (Uc, rc), (Uw, rw) = runs[False], runs[True]
    for r in rc + rw:
        assert r["true_rel_res"] < 1e-10
    assert rc[0]["matvecs"] == rw[0]["matvecs"]
    assert rel_err(Uw, Uc) < 1e-8


_PASS_CHILD = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
from conftest import get_case
from cfdv_b200 import gpu as G
out = {}
for name in sys.argv[3].split(","):
    case = get_case(name)
    with G.FDVSolver(case) as s:
        s.load_node_records()
        s.form(s.cfl(float(case.control["cfl"])), precision=G.PREC_MIXED)
        for prec in (G.PREC_FP64, G.PREC_MIXED):
            for m in (30, 62):
                r = s.gmres(mode=G.GMRES_CORRECT, m=m, restarts=40, rtol=1e-10, precision=prec, engine=0)
                out[f"{name}_{prec}_{m}"] = s.du()
                out[f"{name}_{prec}_{m}_est"] = r["est"]
        # whole steps (formation and solve again each step)
        for k in range(3):
            r = s.step(float(case.control["cfl"]), mode=G.GMRES_CORRECT, m=30, restarts=40, rtol=1e-8,
                       precision=G.PREC_MIXED)
        out[f"{name}_steps"] = s.get_state()
np.savez(sys.argv[2], **out)
"""


def _runs_agree_bitwise(tmp_path, var, names):
    import os
    import subprocess
    import sys
    from conftest import ROOT

    res = {}
    for flag in ("1", "0"):
        out = str(tmp_path / f"{var}{flag}.npz")
        env = dict(os.environ, **{var: flag})
        subprocess.run([sys.executable, "-c", _PASS_CHILD, ROOT, out, ",".join(names)], check=True, env=env,
                       timeout=600)
        res[flag] = dict(np.load(out))
    assert res["1"].keys() == res["0"].keys()
    for k in res["1"]:
        assert np.array_equal(res["1"][k], res["0"][k]), k


def test_3d_element_ring_matches_direct_pass_bitwise(tmp_path):
    """In 3D the mixed form's persistent solve streams the element matrices of every element pass
    (its FP32 products and FP64 restart residuals) through a shared-memory ring of bulk copies;
    CFDV_ELEM_RING=0 selects the pass that loads them directly.  Each row sums in the same order
    in both, so whole solves (mixed, with the FP64 solves beside them, the ring's largest stage
    at m = 30 and a smaller one at m = 62) and whole steps agree bit for bit."""
    _runs_agree_bitwise(tmp_path, "CFDV_ELEM_RING", ["ramp4", "cyl4", "duct4", "ramp4_adap"])
