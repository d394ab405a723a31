"""The adjoint element functionals (cfdv_b200/csrc/adjoint.cuh), built for the CPU by
tests/emu/adj_emu.cpp, against the oracle: the weighted element residual
L_e = w_e . (rhs_e - R_e du_e) against the oracle's formation, its dual-number derivatives
against central finite differences of the oracle's formation, the tangent (JVP) against
the adjoint (VJP) form, and the wall-force functional against closed-form cases."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, SMALL_CASES, get_case

EMU = os.path.join(ROOT, "tests", "emu", "libadj_emu.so")
CSRC = os.path.join(ROOT, "cfdv_b200", "csrc")


@pytest.fixture(scope="module")
def emu():
    src = os.path.join(ROOT, "tests", "emu", "adj_emu.cpp")
    deps = [src] + [os.path.join(CSRC, f) for f in ("adjoint.cuh", "adjoint_warp.cuh", "dual.cuh", "formation.cuh",
                                                     "fdv_physics.cuh", "cfdv_types.h", "jac_adjoint.cuh")]
    if not os.path.exists(EMU) or os.path.getmtime(EMU) < max(os.path.getmtime(f) for f in deps):
        subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-pthread", "-Wno-unknown-pragmas", src, "-o",
                        EMU], check=True)
    L = C.CDLL(EMU)
    P, D, I = C.c_void_p, C.c_double, C.c_int
    L.emu_functional.argtypes = [I, I, P, P, P, P, P, D, D, D, D, D, D, I, D, I, I, P, P, P, D, D, P, P]
    L.emu_wall_force.argtypes = [I, I, P, P, P, P, D, D, D, D, D, D, I, I, P, P]
    L.emu_vjp_warp.argtypes = [I, I, P, P, P, P, P, D, D, D, D, D, D, I, D, I, P, P, P, P, P, P]
    L.emu_set_adaptive.argtypes = [P, P]
    return L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Setup:
    """A case after two textbook steps of the oracle, with seeded weights and dU."""

    def __init__(self, O, name, steps=2):
        self.case = case = get_case(name)
        self.o = o = O.Oracle(case)
        U = o.init_U()
        cl = o.cleng()
        cfl = float(case.control["cfl"])
        for _ in range(steps):
            U = o.step(U, cfl, 20, 5, mode=1, rtol=1e-10, cleng=cl)[0]
        self.U = U
        self.dt = o.cfl(U, cfl, cl)
        rng = np.random.default_rng(20261203)
        self.du = rng.standard_normal(o.n_dof) * 1e-3
        self.w = rng.standard_normal(o.n_dof)
        self.mask = o.rowmask()
        self.x = np.ascontiguousarray(case.nodes[:, : case.ndim])
        self.conn = np.ascontiguousarray(case.conn, np.int32)
        self.bc = np.ascontiguousarray(case.bc, np.int32)
        a = case.aero
        self.gas = (float(a["gamma"]), float(a["M"]), float(a["Re"]), float(a["Pr"]), float(a["Tinf"]),
                    float(a["Twall"]), int(a["Adiabatic"]))
        self.E, self.Ke = case.n_elements, o.Ke
        # adaptive elements: Hnm(N, M) at N + nnod*M
        self.hidx = self.hnm = None
        if case.adap_elements is not None:
            self.hidx = np.ascontiguousarray(case.hnm_index(), np.int32)
            self.hnm = np.ascontiguousarray(np.transpose(case.adap_hnm, (0, 2, 1)), np.float64)

    def arm(self, L):
        """Point the emulator's adaptive-element arrays at this case's (or clear them)."""
        if getattr(self, "hidx", None) is None:
            L.emu_set_adaptive(None, None)
        else:
            L.emu_set_adaptive(_p(self.hidx), _p(self.hnm))

    def idx(self, e):
        nodes = self.case.conn[e]
        return (nodes[:, None] * self.o.neqn + np.arange(self.o.neqn)[None, :]).ravel()

    def emu(self, L, U=None, dt=None, M=None, mode=0, tU=None, tdt=0.0, tM=0.0):
        U = self.U if U is None else U
        dt = self.dt if dt is None else dt
        g = list(self.gas)
        if M is not None:
            g[1] = M
        nd = self.Ke + 2 if mode == 0 else self.Ke
        out = np.zeros(self.E * nd)
        val = np.zeros(self.E)
        tU = self.du if tU is None else tU
        self.arm(L)
        L.emu_functional(self.case.ndim, self.E, _p(U), _p(self.x), _p(self.conn), _p(self.bc), _p(self.mask), *g,
                         float(dt), 0, mode, _p(self.du), _p(self.w), _p(tU), float(tdt), float(tM), _p(out),
                         _p(val))
        return out.reshape(self.E, nd), val

    def oracle_L(self, U=None, dt=None, M=None):
        """w . (rhs - R du) per element over unmasked rows, from the oracle's formation."""
        U = self.U if U is None else U
        dt = self.dt if dt is None else dt
        if M is not None:
            self.o.aero.mach = M
        try:
            R, rhs = self.o.form(U, dt)
        finally:
            self.o.aero.mach = self.gas[1]
        out = np.zeros(self.E)
        for e in range(self.E):
            ix = self.idx(e)
            r = rhs[e] - R[e].T @ self.du[ix]  # R[e, j, i] = R_e(i, j)
            we = self.w[ix].copy()
            for k in range(self.Ke):
                if (int(self.mask[e]) >> k) & 1:
                    we[k] = 0.0
            out[e] = we @ r
        return out


@pytest.mark.parametrize("name", SMALL_CASES + ["lid8_adap", "ramp4_adap"])
def test_functional_value_matches_oracle_residual(emu, oracle_lib, name):
    s = Setup(oracle_lib, name)
    _, val = s.emu(emu)
    ref = s.oracle_L()
    assert np.abs(val - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("name", ["lid8", "plate20", "ramp4", "cyl4", "plate20_adap", "cyl4_adap"])
def test_vjp_matches_finite_differences(emu, oracle_lib, name):
    """Every direction of two elements, and dt and Mach, against central differences of the
    oracle's formation (step 1e-7 relative: the FDV parameter s1 jumps at r = 0.01, so a
    larger step can cross the branch)."""
    s = Setup(oracle_lib, name)
    g, _ = s.emu(emu)
    worst = 0.0
    for e in (s.E // 3, s.E - 1):
        ix = s.idx(e)
        scale = np.abs(g[e]).max()
        for k in range(s.Ke):
            gi = ix[k]
            h = 1e-7 * max(abs(s.U[gi]), 1e-3)
            Up, Um = s.U.copy(), s.U.copy()
            Up[gi] += h
            Um[gi] -= h
            fd = (s.oracle_L(U=Up)[e] - s.oracle_L(U=Um)[e]) / (2 * h)
            worst = max(worst, abs(fd - g[e, k]) / scale)
        h = 1e-7 * s.dt
        fd = (s.oracle_L(dt=s.dt + h)[e] - s.oracle_L(dt=s.dt - h)[e]) / (2 * h)
        # central differences of a residual of size ~scale carry ~1e-16 scale / h of rounding
        assert abs(fd - g[e, s.Ke]) <= 1e-5 * abs(fd) + 1e-7 * scale
        M = s.gas[1]
        h = 1e-7 * M
        fd = (s.oracle_L(M=M + h)[e] - s.oracle_L(M=M - h)[e]) / (2 * h)
        assert abs(fd - g[e, s.Ke + 1]) <= 1e-5 * abs(fd) + 1e-7 * scale
    assert worst <= 1e-5


@pytest.mark.parametrize("name", SMALL_CASES + ["lid8_adap", "ramp4_adap", "cyl4_adap"])
def test_warp_reverse_sweep_matches_forward_mode(emu, oracle_lib, name):
    """The warp reverse sweep (one lane per Gauss point, 32 lanes run here as fibers) against the
    per-seed forward-mode functional: every unknown of every element, d/d dt, d/d Mach and
    the value L_e."""
    s = Setup(oracle_lib, name)
    g, val = s.emu(emu)
    s.arm(emu)
    out = np.zeros(s.E * s.Ke)
    odt, om, ov = np.zeros(s.E), np.zeros(s.E), np.zeros(s.E)
    emu.emu_vjp_warp(s.case.ndim, s.E, _p(s.U), _p(s.x), _p(s.conn), _p(s.bc), _p(s.mask), *s.gas, float(s.dt), 0,
                     _p(s.du), _p(s.w), _p(out), _p(odt), _p(om), _p(ov))
    ref = g[:, : s.Ke]
    assert np.abs(out.reshape(s.E, s.Ke) - ref).max() <= 1e-13 * np.abs(ref).max()
    for got, want in ((odt, g[:, s.Ke]), (ov, val)):
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    # d L_e / d Mach sums terms that cancel: Cv and T both scale with M^-2, so the Cv terms of
    # the Jacobians, the node temperatures and k(M) nearly balance.  On cyl4 one element's
    # terms add up to 18.8 in magnitude for a derivative of 3.8e-8, so both evaluations carry
    # ~1e-16 * 18.8 of rounding; the bound is relative to the largest derivative.
    assert np.abs(om - g[:, s.Ke + 1]).max() <= 1e-11 * np.abs(g[:, s.Ke + 1]).max()


@pytest.mark.parametrize("name", SMALL_CASES)
def test_jvp_is_the_transpose_of_vjp(emu, oracle_lib, name):
    """w . (J t) from the tangent rows equals (J^T w) . t from the adjoint entries."""
    s = Setup(oracle_lib, name)
    rng = np.random.default_rng(7)
    tU = rng.standard_normal(s.o.n_dof) * np.abs(s.U).max() * 1e-2
    tdt, tM = 0.3 * s.dt, 0.05
    g, _ = s.emu(emu)
    jt, _ = s.emu(emu, mode=1, tU=tU, tdt=tdt, tM=tM)
    lhs = rhs = 0.0
    for e in range(s.E):
        ix = s.idx(e)
        we = s.w[ix].copy()
        for k in range(s.Ke):
            if (int(s.mask[e]) >> k) & 1:
                we[k] = 0.0
        lhs += we @ jt[e]
        rhs += g[e, : s.Ke] @ tU[ix] + g[e, s.Ke] * tdt + g[e, s.Ke + 1] * tM
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs))


def _force(emu, s, U, M=None, wall_bc=1):
    g = list(s.gas)
    if M is not None:
        g[1] = M
    Ke = s.Ke
    out = np.zeros(s.E * (Ke + 1))
    val = np.zeros(s.E)
    s.arm(emu)
    emu.emu_wall_force(s.case.ndim, s.E, _p(U), _p(s.x), _p(s.conn), _p(s.bc), *g, int(wall_bc), _p(out), _p(val))
    return out.reshape(s.E, Ke + 1), val


def test_wall_force_plate_shear_closed_form(emu, oracle_lib):
    """u = a y over the plate: only the wall shear acts, F_x = mu(T=1) a L / Re = a L / Re."""
    s = Setup(oracle_lib, "plate20", steps=0)
    a_shear = 0.7
    nodes = s.case.nodes
    U = np.zeros(s.o.n_dof)
    Cv = 1.0 / s.gas[0] / (s.gas[0] - 1.0) / s.gas[1] ** 2
    for n in range(s.case.n_nodes):
        u = a_shear * nodes[n, 1]
        U[4 * n: 4 * n + 4] = [1.0, u, 0.0, Cv * 1.0 + 0.5 * u * u]
    _, val = _force(emu, s, U)
    wall_len = 0.0
    for e in range(s.E):
        for f in range(4):
            if s.case.bc[e, f] == 1:
                p0, p1 = nodes[s.case.conn[e, f], :2], nodes[s.case.conn[e, (f + 1) % 4], :2]
                wall_len += np.hypot(*(p1 - p0))
    assert abs(val.sum() - a_shear * wall_len / s.gas[2]) <= 1e-12 * a_shear * wall_len / s.gas[2]


def test_wall_force_closed_body_uniform_state_vanishes(emu, oracle_lib):
    """A fluid at rest with uniform pressure exerts no net force on the closed cylinder wall."""
    s = Setup(oracle_lib, "cyl4", steps=0)
    U = s.o.init_U()
    U[1::5] = 0.0
    U[2::5] = 0.0
    U[3::5] = 0.0
    U[0::5] = 1.0
    U[4::5] = 1.0
    _, val = _force(emu, s, U)
    ref = np.abs(val).max() * 1.0
    assert abs(val.sum()) <= 1e-13 * max(ref, 1.0)


@pytest.mark.parametrize("name", ["plate20", "cyl4"])
def test_wall_force_gradient_matches_finite_differences(emu, oracle_lib, name):
    s = Setup(oracle_lib, name)
    g, val = _force(emu, s, s.U)
    walls = [e for e in range(s.E) if (s.case.bc[e] == 1).any()]
    assert walls
    for e in walls[:3]:
        ix = s.idx(e)
        scale = np.abs(g[e]).max()
        for k in range(s.Ke):
            # the wall's momentum is zero: the step is taken on the scale of the state, not of
            # the entry, so that rounding does not swamp the difference
            h = 1e-6 * max(abs(s.U[ix[k]]), 1.0)
            Up, Um = s.U.copy(), s.U.copy()
            Up[ix[k]] += h
            Um[ix[k]] -= h
            fd = (_force(emu, s, Up)[1][e] - _force(emu, s, Um)[1][e]) / (2 * h)
            assert abs(fd - g[e, k]) <= 1e-6 * scale
        M = s.gas[1]
        h = 1e-7 * M
        fd = (_force(emu, s, s.U, M + h)[1][e] - _force(emu, s, s.U, M - h)[1][e]) / (2 * h)
        assert abs(fd - g[e, s.Ke]) <= 1e-6 * max(abs(fd), scale)
