"""The formation kernel's phases (cfdv_b200/csrc/formation.cuh), run thread by thread
on the CPU by tests/emu/form_emu.cpp, against the oracle.  This checks the kernel's
index arithmetic and factored contraction without a GPU."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, SMALL_CASES, get_case, rel_err, elem_rel_err

EMU = os.path.join(ROOT, "tests", "emu", "libform_emu.so")


@pytest.fixture(scope="module")
def emu():
    src = os.path.join(ROOT, "tests", "emu", "form_emu.cpp")
    if not os.path.exists(EMU) or os.path.getmtime(EMU) < max(
            os.path.getmtime(src), *[os.path.getmtime(os.path.join(ROOT, "cfdv_b200", "csrc", f))
                                     for f in ("formation.cuh", "fdv_physics.cuh", "cfdv_types.h")]):
        subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wno-unknown-pragmas", src, "-o", EMU],
                       check=True)
    L = C.CDLL(EMU)
    P, D, I = C.c_void_p, C.c_double, C.c_int
    L.emu_form.argtypes = [I, I, P, P, P, P, P, D, D, D, D, D, D, I, D, I, P, P, P, P]
    L.emu_set_adaptive.argtypes = [P, P]
    return L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def run_emu(L, case, U, dt, mask, phys=0):
    E, Ke = case.n_elements, case.nnod * case.neqn
    R = np.zeros((E, Ke, Ke))
    R32 = np.zeros((E, Ke, Ke), np.float32)
    rhs = np.zeros((E, Ke))
    s = np.zeros((E, 4))
    x = np.ascontiguousarray(case.nodes[:, : case.ndim])
    conn = np.ascontiguousarray(case.conn, np.int32)
    bc = np.ascontiguousarray(case.bc, np.int32)
    a = case.aero
    bad = L.emu_form(case.ndim, E, _p(U), _p(x), _p(conn), _p(bc), _p(mask), float(a["gamma"]), float(a["M"]),
                     float(a["Re"]), float(a["Pr"]), float(a["Tinf"]), float(a["Twall"]), int(a["Adiabatic"]),
                     dt, phys, _p(R), _p(R32), _p(rhs), _p(s))
    return bad, R, R32, rhs, s


@pytest.mark.parametrize("name", SMALL_CASES)
@pytest.mark.parametrize("phys", [0, 1])
def test_emulated_formation_matches_oracle(emu, oracle_lib, name, phys):
    case = get_case(name)
    if phys and case.ndim == 2:
        pytest.skip("the 3D flux switch has no effect in 2D")
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    dt = o.cfl(U, float(case.control["cfl"]))
    Ro, ro = o.form(U, dt, apply_bc=True, physical_3d_flux=bool(phys))
    bad, R, R32, rhs, s = run_emu(emu, case, U, dt, o.rowmask(), phys)
    assert bad == 0
    assert elem_rel_err(R, Ro) <= 1e-13
    assert rel_err(rhs, ro) <= 1e-13
    assert rel_err(s, o.fdvparam(U)) == 0.0
    assert elem_rel_err(R32.astype(np.float64), Ro) <= 1e-6


@pytest.mark.parametrize("name", SMALL_CASES)
def test_emulated_adaptive_formation_matches_oracle(emu, oracle_lib, name):
    """Adaptive (hanging-node) elements: every third element carries an Hnm; the kernel's
    phases against the oracle restatement (itself pinned to the reference's outputs on the
    same cases, tests/golden/*_adap.npz)."""
    from cfdv_b200 import meshgen as mg
    case = mg.adaptive_demo(get_case(name))
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    dt = o.cfl(U, float(case.control["cfl"]))
    Ro, ro = o.form(U, dt, apply_bc=True)
    idx = np.ascontiguousarray(case.hnm_index(), np.int32)
    hnm = np.ascontiguousarray(np.transpose(case.adap_hnm, (0, 2, 1)), np.float64)  # Hnm(N, M) at N + nnod*M
    emu.emu_set_adaptive(_p(idx), _p(hnm))
    try:
        bad, R, R32, rhs, s = run_emu(emu, case, U, dt, o.rowmask())
    finally:
        emu.emu_set_adaptive(None, None)
    assert bad == 0
    assert elem_rel_err(R, Ro) <= 1e-13
    assert rel_err(rhs, ro) <= 1e-13
    plain = oracle_lib.Oracle(get_case(name)).form(U, dt, apply_bc=True)[0]
    assert elem_rel_err(R[case.adap_elements], plain[case.adap_elements]) > 1e-6  # the transform acted
