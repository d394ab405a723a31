"""Discrete adjoint and tangent of the step on the GPU (through the C ABI).

* The element functionals run by the CUDA kernels agree with the same functionals built
  for the CPU (tests/emu/adj_emu.cpp), which tests/test_adjoint_emulated.py checks
  against the oracle and finite differences.
* The adjoint gradient of J = mean_{n=1..N} F_x(U_n) agrees with the FP64 tangent-linear
  run along the same parameter directions (both are exact derivatives of the same
  discrete map, so they agree to the solve tolerance: 1e-8 relative here).
* It agrees with central finite differences, step 1e-6 relative, of the GPU's own FP64
  forward run and of the oracle's CPU solve (the restatement pinned to the reference,
  textbook mode), to 1e-5 relative, for the Mach number and the wall temperature; single
  wall nodes are checked against unit tangent runs (see the test for why).
* Checkpoint spacing does not change the gradient; the mixed-precision adjoint agrees
  with FP64 to 1e-6."""
import numpy as np
import pytest

from conftest import get_case
from test_adjoint_emulated import Setup, _force, _p

pytestmark = pytest.mark.gpu

ADJ_CASE = "cyl4"     # the O-grid cylinder with an isothermal wall (bc 1)
N_STEPS, CFL, M_GMRES, RTOL = 6, 0.5, 40, 1e-12


@pytest.fixture(scope="module")
def gpu():
    from cfdv_b200 import gpu as G
    return G


@pytest.fixture(scope="module")
def emu():
    return _load_emu()


def _load_emu():
    import ctypes as C
    import os
    import subprocess
    from conftest import ROOT
    src = os.path.join(ROOT, "tests", "emu", "adj_emu.cpp")
    lib = os.path.join(ROOT, "tests", "emu", "libadj_emu.so")
    if not os.path.exists(lib):
        subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wno-unknown-pragmas", src, "-o", lib],
                       check=True)
    L = C.CDLL(lib)
    P, D, I = C.c_void_p, C.c_double, C.c_int
    L.emu_functional.argtypes = [I, I, P, P, P, P, P, D, D, D, D, D, D, I, D, I, I, P, P, P, D, D, P, P]
    L.emu_wall_force.argtypes = [I, I, P, P, P, P, D, D, D, D, D, D, I, I, P, P]
    L.emu_set_element_mask.argtypes = [P]
    L.emu_set_adaptive.argtypes = [P, P]
    return L


def gather(s, rows):
    """Node vector sum_e P_e^T rows_e from per-element rows [E][Ke]."""
    g = np.zeros(s.o.n_dof)
    for e in range(s.E):
        np.add.at(g, s.idx(e), rows[e])
    return g


# The lid's cell Reynolds numbers are small enough that the reference's SUPG coefficient
# coth(R/2) - 2/R (FDVGalerkin.h:46-50) keeps only a few significant digits: moving cosh up
# and sinh down by two ulps in the CPU build shifts its assembled gradient by 1.4e-4 and its
# tangent by 1.2e-4 relative (values by 1.4e-10), and CUDA's cosh/sinh are not glibc's.  The
# other cases, and the 3D path (no SUPG term), agree to rounding.
TOL_VAL = {"lid8": 1e-9}
TOL_DER = {"lid8": 1e-3}


@pytest.mark.parametrize("name", ["lid8", "plate20", "ramp4", "cyl4", "plate20_adap", "cyl4_adap"])
def test_functionals_match_cpu_build(gpu, emu, oracle_lib, name):
    s = Setup(oracle_lib, name)
    with gpu.FDVSolver(s.case) as g:
        g.set_state(s.U)
        g.form(s.dt)
        L = g.element_functional(s.w, s.du)
        gU, gdt, gm = g.vjp(s.w, s.du)
        rng = np.random.default_rng(3)
        tU = rng.standard_normal(s.o.n_dof) * np.abs(s.U).max() * 1e-2
        dr = g.jvp(s.du, tU, 0.2 * s.dt, 0.01)
        walls = (s.case.bc == 1).any()
        F = g.wall_force(1, grad=True) if walls else None
    tv, td = TOL_VAL.get(name, 1e-11), TOL_DER.get(name, 1e-10)
    ge, Le = s.emu(emu)
    assert np.abs(L - Le).max() <= tv * np.abs(Le).max()
    ref = gather(s, ge[:, : s.Ke])
    assert np.abs(gU - ref).max() <= td * np.abs(ref).max()
    assert gdt == pytest.approx(ge[:, s.Ke].sum(), rel=td, abs=1e-12 * np.abs(ge[:, s.Ke]).max())
    assert gm == pytest.approx(ge[:, s.Ke + 1].sum(), rel=td, abs=1e-12 * np.abs(ge[:, s.Ke + 1]).max())
    je, _ = s.emu(emu, mode=1, tU=tU, tdt=0.2 * s.dt, tM=0.01)
    jref = gather(s, je)
    assert np.abs(dr - jref).max() <= td * np.abs(jref).max()
    if F is not None:
        fe, fv = _force(emu, s, s.U)
        assert F[0] == pytest.approx(fv.sum(), rel=1e-12)
        fref = gather(s, fe[:, : s.Ke])
        assert np.abs(F[1] - fref).max() <= 1e-10 * np.abs(fref).max()
        assert F[2] == pytest.approx(fe[:, s.Ke].sum(), rel=1e-10)


def _solver(G, case):
    s = G.FDVSolver(case)
    s.load_node_records()
    return s


@pytest.fixture(scope="module")
def adj(gpu):
    case = get_case(ADJ_CASE)
    with _solver(gpu, case) as s:
        r = s.adjoint(N_STEPS, CFL, checkpoint_every=2, m=M_GMRES, rtol=RTOL)
    assert len(r["wall_nodes"]) > 0
    return r


def test_adjoint_matches_tangent_linear(gpu, adj):
    case = get_case(ADJ_CASE)
    rng = np.random.default_rng(11)
    v = rng.standard_normal(len(adj["wall_nodes"]))
    with _solver(gpu, case) as s:
        J, dJm = s.tangent(N_STEPS, CFL, dmach=1.0, m=M_GMRES, rtol=RTOL)
        J2, dJt = s.tangent(N_STEPS, CFL, dT_wall=v, m=M_GMRES, rtol=RTOL)
    assert J == pytest.approx(adj["J"], rel=1e-12)
    assert J2 == pytest.approx(adj["J"], rel=1e-12)
    assert adj["dJ_dmach"] == pytest.approx(dJm, rel=1e-8)
    assert float(adj["dJ_dtnode"] @ v) == pytest.approx(dJt, rel=1e-8)
    assert adj["dJ_dtwall"] == pytest.approx(adj["dJ_dtnode"].sum(), rel=1e-14)


def _with_mach(case, M):
    import copy
    c = copy.deepcopy(case)
    c.aero = dict(case.aero)
    c.aero["M"] = M
    return c


def _with_wall_T(case, wall, dT):
    import copy
    c = copy.deepcopy(case)
    c.nodes = case.nodes.copy()
    c.nodes[wall, 2 * case.ndim + 1] += dT
    return c


def _gpu_J(G, case):
    with _solver(G, case) as s:
        J, _ = s.tangent(N_STEPS, CFL, dmach=0.0, m=M_GMRES, rtol=RTOL)
    return J


def test_adjoint_matches_gpu_finite_differences(gpu, adj):
    case = get_case(ADJ_CASE)
    M = float(case.aero["M"])
    h = 1e-6 * M
    fd = (_gpu_J(gpu, _with_mach(case, M + h)) - _gpu_J(gpu, _with_mach(case, M - h))) / (2 * h)
    assert adj["dJ_dmach"] == pytest.approx(fd, rel=1e-5)
    wall = adj["wall_nodes"]
    h = 1e-6
    fd = (_gpu_J(gpu, _with_wall_T(case, wall, h)) - _gpu_J(gpu, _with_wall_T(case, wall, -h))) / (2 * h)
    assert adj["dJ_dtwall"] == pytest.approx(fd, rel=1e-5)


def test_per_node_gradient_matches_unit_tangents(gpu, adj):
    """Single wall nodes are checked against tangent runs along unit directions, not against
    differences: the wall starts at rest at one temperature, so the CFL minimum
    (MPI_CFL.h:7-56) is attained at many wall nodes at once, and moving one node's
    temperature breaks the tie on one side only (dt = cfl * min is not differentiable
    there).  Both the adjoint and the tangent give the whole dt sensitivity to the first
    arg-min node in element order."""
    case = get_case(ADJ_CASE)
    g = adj["dJ_dtnode"]
    picks = {int(np.argmax(np.abs(g))), int(np.argmin(np.abs(g))), len(g) // 2}
    with _solver(gpu, case) as s:
        for k in sorted(picks):
            e = np.zeros(len(g))
            e[k] = 1.0
            _, dJ = s.tangent(N_STEPS, CFL, dT_wall=e, m=M_GMRES, rtol=RTOL)
            assert g[k] == pytest.approx(dJ, rel=1e-8, abs=1e-10 * np.abs(g).max())


def _oracle_J(O, emu, case):
    """J of the oracle's textbook-mode CPU solve, with the wall force of the CPU build."""
    s = Setup.__new__(Setup)
    s.case = case
    s.o = o = O.Oracle(case)
    s.x = np.ascontiguousarray(case.nodes[:, : case.ndim])
    s.conn = np.ascontiguousarray(case.conn, np.int32)
    s.bc = np.ascontiguousarray(case.bc, np.int32)
    a = case.aero
    s.gas = (float(a["gamma"]), float(a["M"]), float(a["Re"]), float(a["Pr"]), float(a["Tinf"]), float(a["Twall"]),
             int(a["Adiabatic"]))
    s.E, s.Ke = case.n_elements, o.Ke
    U = o.init_U()
    cl = o.cleng()
    J = 0.0
    for _ in range(N_STEPS):
        U = o.step(U, CFL, M_GMRES, 200, mode=1, rtol=RTOL, cleng=cl)[0]
        J += _force(emu, s, U)[1].sum()
    return J / N_STEPS


def test_adjoint_matches_oracle_finite_differences(emu, oracle_lib, adj):
    case = get_case(ADJ_CASE)
    M = float(case.aero["M"])
    h = 1e-6 * M
    assert _oracle_J(oracle_lib, emu, case) == pytest.approx(adj["J"], rel=1e-10)
    fd = (_oracle_J(oracle_lib, emu, _with_mach(case, M + h)) -
          _oracle_J(oracle_lib, emu, _with_mach(case, M - h))) / (2 * h)
    assert adj["dJ_dmach"] == pytest.approx(fd, rel=1e-5)
    wall = adj["wall_nodes"]
    h = 1e-6
    fd = (_oracle_J(oracle_lib, emu, _with_wall_T(case, wall, h)) -
          _oracle_J(oracle_lib, emu, _with_wall_T(case, wall, -h))) / (2 * h)
    assert adj["dJ_dtwall"] == pytest.approx(fd, rel=1e-5)


def test_checkpoint_spacing_and_mixed_precision(gpu, adj):
    case = get_case(ADJ_CASE)
    with _solver(gpu, case) as s:
        r1 = s.adjoint(N_STEPS, CFL, checkpoint_every=1, m=M_GMRES, rtol=RTOL)
        rN = s.adjoint(N_STEPS, CFL, checkpoint_every=N_STEPS, m=M_GMRES, rtol=RTOL)
        s.load_node_records()
        rm = s.adjoint(N_STEPS, CFL, checkpoint_every=3, m=M_GMRES, rtol=1e-10, precision=gpu.PREC_MIXED)
    # the recomputed steps' element matrices and each segment's last step's (from the forward
    # run) stay on the device for their reverse steps: none forms again when they all fit
    assert (adj["kept_matrix_sets"], adj["reverse_forms"]) == (1 + 3, 0)
    assert (r1["kept_matrix_sets"], r1["reverse_forms"]) == (N_STEPS, 0)
    assert (rN["kept_matrix_sets"], rN["reverse_forms"]) == (N_STEPS - 1 + 1, 0)
    assert (rm["kept_matrix_sets"], rm["reverse_forms"]) == (2 + 2, 0)
    for r in (r1, rN):
        assert r["dJ_dmach"] == pytest.approx(adj["dJ_dmach"], rel=1e-13)
        assert np.abs(r["dJ_dtnode"] - adj["dJ_dtnode"]).max() <= 1e-13 * np.abs(adj["dJ_dtnode"]).max()
    # mixed precision: the same gradient to 1e-6 (its states differ from FP64 by ~1e-10, which
    # can move the CFL tie to another wall node: that moves the dt share, ~1e-5 of the
    # largest entry, between tied nodes and leaves the totals unchanged)
    assert rm["dJ_dmach"] == pytest.approx(adj["dJ_dmach"], rel=1e-6)
    assert rm["dJ_dtwall"] == pytest.approx(adj["dJ_dtwall"], rel=1e-6)
    assert np.abs(rm["dJ_dtnode"] - adj["dJ_dtnode"]).max() <= 1e-4 * np.abs(adj["dJ_dtnode"]).max()


def test_kept_matrix_sets_change_nothing(gpu, adj):
    """The same gradient whether the reverse steps form their matrices again (no kept sets), keep
    the recomputed steps' only (one set at k = 2) or keep all (to 1e-13: a kept set was formed
    inside a step, with dt^2/2 from the device's dt, a re-formed one with the host's)."""
    case = get_case(ADJ_CASE)
    with _solver(gpu, case) as s:
        r0 = s.adjoint(N_STEPS, CFL, checkpoint_every=2, m=M_GMRES, rtol=RTOL, max_kept_sets=-1)
        s.load_node_records()
        r1 = s.adjoint(N_STEPS, CFL, checkpoint_every=2, m=M_GMRES, rtol=RTOL, max_kept_sets=1)
    assert (r0["kept_matrix_sets"], r0["reverse_forms"]) == (0, N_STEPS)
    assert (r1["kept_matrix_sets"], r1["reverse_forms"]) == (1, 3)
    for r in (r0, r1):
        assert r["dJ_dmach"] == pytest.approx(adj["dJ_dmach"], rel=1e-13)
        assert r["dJ_dtwall"] == pytest.approx(adj["dJ_dtwall"], rel=1e-13)
        assert np.abs(r["dJ_dtnode"] - adj["dJ_dtnode"]).max() <= 1e-13 * np.abs(adj["dJ_dtnode"]).max()


def test_vjp_full_size_cylinder_sampled(gpu, emu, oracle_lib):
    """The reverse sweep on the full cylinder 96x128x16 (184,320 hex8, the adjoint leg's mesh)
    after two FP64 steps: adjoint weights on the nodes of sampled elements only (interior, and
    the first and last element with each pattern of boundary codes: wall, far field, symmetry
    planes), so that exactly the elements touching those nodes contribute.  The GPU's assembled
    gradient, d/d dt and d/d M against the forward-mode functional of the CPU build over those
    elements."""
    from cfdv_b200 import meshgen as mg
    case = mg.FULL["cylinder"]()
    o = oracle_lib.Oracle(case)
    E, nnod, neqn, Ke = case.n_elements, 8, 5, 40
    conn = np.ascontiguousarray(case.conn, np.int32)
    bc = np.ascontiguousarray(case.bc, np.int32)
    rng = np.random.default_rng(20261204)
    pick = set(rng.choice(E, 6, replace=False).tolist())
    pats = {}
    for e, row in enumerate(map(tuple, bc)):
        if any(row):
            pats.setdefault(row, []).append(e)
    for es in pats.values():
        pick.update((es[0], es[-1]))
    nodes = np.unique(conn[sorted(pick)].ravel())
    w = np.zeros(case.n_nodes * neqn)
    for q in range(neqn):
        w[nodes * neqn + q] = rng.standard_normal(len(nodes))
    du = rng.standard_normal(case.n_nodes * neqn) * 1e-3
    cfl = float(case.control["cfl"])
    with gpu.FDVSolver(case) as s:
        s.set_state(o.init_U())
        for _ in range(2):
            s.step(cfl, mode=gpu.GMRES_CORRECT, m=40, restarts=20, rtol=1e-10)
        U = s.get_state()
        dt = s.cfl(cfl)
        s.form(dt)
        gU, gdt, gm = s.vjp(w, du)
    touched = np.isin(conn, nodes).any(axis=1)
    mask = np.ascontiguousarray(touched.astype(np.uint8))
    x = np.ascontiguousarray(case.nodes[:, :3])
    rm = o.rowmask()
    a = case.aero
    gas = (float(a["gamma"]), float(a["M"]), float(a["Re"]), float(a["Pr"]), float(a["Tinf"]), float(a["Twall"]),
           int(a["Adiabatic"]))
    out = np.zeros(E * (Ke + 2))
    val = np.zeros(E)
    emu.emu_set_adaptive(None, None)
    emu.emu_set_element_mask(_p(mask))
    try:
        emu.emu_functional(3, E, _p(U), _p(x), _p(conn), _p(bc), _p(rm), *gas, float(dt), 0, 0, _p(du), _p(w),
                           _p(du), 0.0, 0.0, _p(out), _p(val))
    finally:
        emu.emu_set_element_mask(None)
    rows = out.reshape(E, Ke + 2)
    ref = np.zeros(case.n_nodes * neqn)
    for e in np.nonzero(touched)[0]:
        ix = (conn[e][:, None] * neqn + np.arange(neqn)[None, :]).ravel()
        np.add.at(ref, ix, rows[e, :Ke])
    assert touched.sum() >= 6 * 8 and len(pats) >= 3
    assert np.abs(gU - ref).max() <= 1e-10 * np.abs(ref).max()
    assert gdt == pytest.approx(rows[:, Ke].sum(), rel=1e-10)
    # the Mach derivative sums terms that nearly cancel (Cv and T both scale with M^-2)
    assert gm == pytest.approx(rows[:, Ke + 1].sum(), rel=1e-8, abs=1e-11 * np.abs(rows[:, Ke + 1]).max())
