"""CUDA path (through the C ABI) against the oracle and the reference's golden outputs.

Tolerances: element matrices, rhs and the EBE product agree with the FP64 oracle to
<= 1e-12 relative (per element max-norm); the reference-mode solve, whose break
decisions and Givens arithmetic run on the host exactly as in the reference, matches
the per-step GMRES history and conserved fields to <= 1e-10 relative (the parity bar
for the plain FP64 form); the textbook solver reaches its 1e-8 true residual in FP64 and in mixed
precision, the mixed field within 1e-6 of FP64."""
import numpy as np
import pytest

from conftest import ADAPTIVE_CASES, SMALL_CASES, get_case, golden, rel_err, elem_rel_err

pytestmark = pytest.mark.gpu

# Element matrices: max-norm error per element relative to that element's max entry;
# rhs vectors: relative to the global max (uniform-state elements carry roundoff-only rhs).
TOL_R = {name: 1e-12 for name in SMALL_CASES + ADAPTIVE_CASES}
# The reference's final estimate g(m) on the stiff cylinder case moves by 3e-7 of itself
# (2.6e-8 of the history scale) under rounding-level changes of the element rhs: the
# formation kernel run on the CPU with FMA contraction reproduces exactly this shift while
# U stays within 6.5e-11, and the reference compiled with FMA changes its own iteration
# count (26 -> 28) and dU by 80%.  The bound below is that measured envelope.
TOL_GFINAL = {"cyl4": 1e-6, "cyl4_adap": 1e-6}
# Same case, later steps: the reference-mode solve (near-diagonal back substitution, no
# restart to a tolerance) carries those differences into the next step's history.  With
# the GPU's arithmetic reproduced on the CPU (tests/emu built with FMA contraction) the
# cylinder's estimate history moves by 2.0e-8 and U by 1.5e-7 after two steps; every
# other case stays below 1e-13.
TOL_HIST = {"cyl4": 1e-7, "cyl4_adap": 1e-7}
TOL_U = {"cyl4": 1e-6, "cyl4_adap": 1e-6}
# The per-field RMS change sqrt(sum U^2 / sum U0^2) - 1 of the cylinder's z-momentum (a
# field that starts at zero and stays small) amplifies those U differences: the GPU's
# arithmetic reproduced on the CPU moves the step-1 RMS vector by 0.063 of its max, the GPU
# by 0.070, and the reference itself, built with FMA contraction, by 0.51 (U by 7.4e-5).
TOL_RMS = {"cyl4": 0.1, "cyl4_adap": 0.1}


@pytest.fixture(scope="module")
def gpu():
    from cfdv_b200 import gpu as G
    return G


def solver(G, case, **kw):
    s = G.FDVSolver(case, **kw)
    s.load_node_records()
    return s


@pytest.mark.parametrize("name", SMALL_CASES + ADAPTIVE_CASES)
def test_formation_matches_oracle(gpu, oracle_lib, name):
    case = get_case(name)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    with solver(gpu, case) as s:
        assert rel_err(s.get_state(), U) == 0.0
        cfl = float(case.control["cfl"])
        dt = s.cfl(cfl)
        assert dt == pytest.approx(o.cfl(U, cfl), rel=1e-14)
        s.form(dt)
        R, rhs = s.element_matrices()
        sp = s.fdv_params()
    Ro, ro = o.form(U, dt, apply_bc=True)
    assert elem_rel_err(R, Ro) <= TOL_R[name]
    assert rel_err(rhs, ro) <= TOL_R[name]
    assert rel_err(sp, o.fdvparam(U)) <= 1e-14


@pytest.mark.parametrize("name", SMALL_CASES + ADAPTIVE_CASES)
def test_formation_matches_reference_golden(gpu, name):
    g, case = golden(name), get_case(name)
    with solver(gpu, case) as s:
        s.form(float(g["dt_dump"][0]))
        R, rhs = s.element_matrices()
    el = g["elements"]
    assert elem_rel_err(R[el], g["R_bc"]) <= TOL_R[name]
    assert rel_err(rhs[el], g["rhs_bc"]) <= TOL_R[name]


@pytest.mark.parametrize("name", ["lid8", "ramp4"])
def test_physical_3d_flux_switch(gpu, oracle_lib, name):
    case = get_case(name)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    with solver(gpu, case, physical_3d_flux=True) as s:
        dt = s.cfl(0.25)
        s.form(dt)
        R, rhs = s.element_matrices()
    Ro, ro = o.form(U, dt, apply_bc=True, physical_3d_flux=True)
    assert elem_rel_err(R, Ro) <= 1e-12 and rel_err(rhs, ro) <= 1e-12


@pytest.mark.parametrize("name", SMALL_CASES)
def test_ebe_product_and_rhs(gpu, oracle_lib, name):
    case = get_case(name)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    rng = np.random.default_rng(7)
    x = rng.standard_normal(o.n_dof)
    with solver(gpu, case) as s:
        dt = s.cfl(float(case.control["cfl"]))
        s.form(dt, precision=gpu.PREC_MIXED)
        y = s.matvec(x)
        yt = s.matvec(x, transpose=True)
        y32 = s.matvec(x, precision=gpu.PREC_MIXED)
        b = s.rhs_vector()
    Ro, ro = o.form(U, dt)
    assert rel_err(y, o.matvec(Ro, x)) <= 1e-12
    assert rel_err(yt, o.matvec(Ro, x, transpose=True)) <= 1e-12
    assert rel_err(y32, o.matvec(Ro, x)) <= 1e-5
    assert rel_err(b, o.compose_rhs(ro)) <= 1e-13


@pytest.mark.parametrize("name", SMALL_CASES + ADAPTIVE_CASES)
def test_reference_gmres_matches_golden_history(gpu, name):
    g, case = golden(name), get_case(name)
    m, r, cfl = int(case.control["gmresiter"]), int(case.control["gmresrestart"]), float(case.control["cfl"])
    with solver(gpu, case) as s:
        for k in range(int(g["steps"])):
            rep = s.step(cfl, mode=gpu.GMRES_REFERENCE, m=m, restarts=r)
            assert rep["dt"] == pytest.approx(g[f"dt@{k}"][0], rel=1e-12)
            assert rep["tol"] == pytest.approx(g[f"tol@{k}"][0], rel=1e-12)
            assert len(rep["est"]) == len(g[f"est@{k}"])
            assert rel_err(rep["est"], g[f"est@{k}"]) <= TOL_HIST.get(name, 1e-10)
            # g(m) is the converged estimate: compare it on the history's scale (~||r0||)
            scale = np.abs(g[f"est@{k}"]).max()
            assert np.abs(rep["gfinal"] - g[f"gfinal@{k}"]).max() <= TOL_GFINAL.get(name, 1e-10) * scale
            assert rel_err(s.get_state(), g[f"U@{k}"]) <= TOL_U.get(name, 1e-10)
            assert rel_err(s.rms(), g[f"rms@{k}"]) <= TOL_RMS.get(name, 1e-7)


def test_reference_mode_long_run_lid32(gpu, oracle_lib):
    """Configuration 1 (lid-driven cavity 32x32, GMRES(20), CFL 0.5): 200 steps of the
    reference solver on the GPU vs the oracle, conserved fields and GMRES history."""
    from cfdv_b200 import meshgen as mg
    case = mg.lid(32)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    cl = o.cleng()
    worst_est = 0.0
    with solver(gpu, case) as s:
        for k in range(200):
            rep = s.step(0.5, mode=gpu.GMRES_REFERENCE, m=20, restarts=1)
            U, _, dt, rms, orep = o.step(U, 0.5, 20, 1, mode=0, cleng=cl)
            assert len(rep["est"]) == len(orep["est"])
            worst_est = max(worst_est, rel_err(rep["est"], orep["est"]))
        Ug = s.get_state()
    assert worst_est <= 1e-10
    assert rel_err(Ug, U) <= 1e-10


@pytest.mark.parametrize("name", ["lid8", "plate20", "ramp4", "duct4"])
def test_correct_gmres_fp64_and_mixed(gpu, oracle_lib, name):
    case = get_case(name)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    with solver(gpu, case) as s:
        dt = s.cfl(float(case.control["cfl"]))
        s.form(dt, precision=gpu.PREC_MIXED)
        r64 = s.gmres(mode=gpu.GMRES_CORRECT, m=30, restarts=60, rtol=1e-8)
        du64 = s.du()
        r32 = s.gmres(mode=gpu.GMRES_CORRECT, m=30, restarts=60, rtol=1e-8, precision=gpu.PREC_MIXED)
        du32 = s.du()
    assert r64["true_rel_res"] < 1e-8
    assert r32["true_rel_res"] < 1e-8
    Ro, ro = o.form(U, dt)
    b = o.compose_rhs(ro)
    res = np.linalg.norm(b - o.matvec(Ro, du64)) / np.linalg.norm(b)
    assert res < 1e-8
    duo, _ = o.gmres_correct(Ro, ro, 30, 60, 1e-12)
    assert rel_err(du64, duo) <= 1e-6
    assert rel_err(du32, du64) <= 1e-6


@pytest.mark.parametrize("name", ["lid8", "plate20", "ramp4", "cyl4", "ramp4_adap"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("orth", ["cgs2", "mgs", "dcgs2"])
def test_persistent_engine_matches_host_driven(gpu, name, prec, orth):
    """The single-launch cooperative solve, with either orthogonalisation, against the
    one-kernel-per-pass MGS solve: same stopping point, same solution to the tolerance."""
    case = get_case(name)
    p = gpu.PREC_MIXED if prec == "mixed" else gpu.PREC_FP64
    with solver(gpu, case) as s:
        dt = s.cfl(float(case.control["cfl"]))
        s.form(dt, precision=gpu.PREC_MIXED)
        r0 = s.gmres(mode=gpu.GMRES_CORRECT, m=30, restarts=80, rtol=1e-8, precision=p, engine=0,
                     orth={"cgs2": 0, "mgs": 1, "dcgs2": 2}[orth])
        d0 = s.du()
        r1 = s.gmres(mode=gpu.GMRES_CORRECT, m=30, restarts=80, rtol=1e-8, precision=p, engine=1)
        d1 = s.du()
    assert r0["true_rel_res"] < 1e-8 and r1["true_rel_res"] < 1e-8
    assert rel_err(d0, d1) <= 1e-6
    assert r0["restarts"] == r1["restarts"]
    # the Givens estimates of the two Arnoldi processes agree to rounding of the basis
    n = min(len(r0["est"]), len(r1["est"]))
    assert abs(len(r0["est"]) - len(r1["est"])) <= 1
    assert rel_err(np.abs(r0["est"][:n]), np.abs(r1["est"][:n])) <= 1e-6


@pytest.mark.parametrize("name", ["lid8", "ramp4", "cyl4"])
def test_solver_plugin_with_host_matrices(gpu, oracle_lib, name):
    """GMRESbase-only use: matrices formed on the CPU (the oracle stands in for the
    reference's FDVGalerkin), uploaded, and solved by the reference-mode GPU GMRES."""
    case = get_case(name)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    dt = o.cfl(U, float(case.control["cfl"]))
    R, rhs = o.form(U, dt)
    m, r = int(case.control["gmresiter"]), int(case.control["gmresrestart"])
    du_o, rep_o = o.gmres_ref(R, rhs, m, r)
    with solver(gpu, case) as s:
        s.set_element_matrices(R, rhs)
        rep = s.gmres(mode=gpu.GMRES_REFERENCE, m=m, restarts=r)
        du = s.du()
    assert len(rep["est"]) == len(rep_o["est"])
    assert rel_err(rep["est"], rep_o["est"]) <= 1e-10
    assert rel_err(du, du_o) <= 1e-10
