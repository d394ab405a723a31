"""Python access to the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``oracle/libcfdv_oracle.so`` (the restatement, ``cfdv_oracle.cpp``) through
ctypes, and reads the record files written by the reference build
(``oracle/_ref/cfdv_ref``, see ``ref_driver.cpp``).  Only tests/, smoke() and
bench.py's CPU-baseline leg import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcfdv_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "cfdv_ref")

_lib = None


# The reference checkout: CFDV_REFERENCE_SRC, else a "reference" tree beside this repository.
REF_SRC_DEFAULT = os.path.normpath(os.path.join(HERE, "..", "..", "reference", "src"))


def build(quiet: bool = True) -> None:
    """Compile the restatement (and the reference build when its sources are present)."""
    subprocess.run(["make", "-C", HERE, "port"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)
    ref_src = os.environ.get("CFDV_REFERENCE_SRC", REF_SRC_DEFAULT)
    if os.path.isdir(ref_src):
        subprocess.run(["make", "-C", HERE, "ref", f"REF={ref_src}"], check=True,
                       stdout=subprocess.DEVNULL if quiet else None)
        # the reference loop with the B200 plug-ins, once the CUDA library is built
        if os.path.exists(os.path.join(HERE, "..", "cfdv_b200", "libcfdv_gpu.so")):
            subprocess.run(["make", "-C", HERE, "ref-gpu", f"REF={ref_src}"], check=True,
                           stdout=subprocess.DEVNULL if quiet else None)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.oracle_dirichlet.argtypes = [P, P, P]
        L.oracle_bc_rowmask.argtypes = [P, P, P, P]
        L.oracle_init_U.argtypes = [P, P, P, P]
        L.oracle_cleng.argtypes = [P, P]
        L.oracle_cfl.argtypes = [P, P, P, P, C.c_double]
        L.oracle_cfl.restype = C.c_double
        L.oracle_fdvparam.argtypes = [P, P, P, P]
        L.oracle_form.argtypes = [P, P, P, C.c_double, C.c_int, C.c_int, P, P]
        L.oracle_compose_rhs.argtypes = [P, P, P]
        L.oracle_ebe_matvec.argtypes = [P, P, P, P]
        L.oracle_ebe_matvec_t.argtypes = [P, P, P, P]
        L.oracle_gmres_ref.argtypes = [P, P, P, C.c_int, C.c_int, P, P]
        L.oracle_gmres_correct.argtypes = [P, P, P, C.c_int, C.c_int, C.c_double, P, P]
        L.oracle_step.argtypes = [P, P, P, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                                  P, P, P, P, P]
        L.oracle_gauss.argtypes = [C.c_int, P, P]
        _lib = L
    return _lib


class _Mesh(C.Structure):
    _fields_ = [("ndim", C.c_int), ("nnod", C.c_int), ("neqn", C.c_int), ("nbnod", C.c_int),
                ("nface", C.c_int), ("n_nodes", C.c_int), ("n_elements", C.c_int),
                ("x", C.c_void_p), ("conn", C.c_void_p), ("bc", C.c_void_p),
                ("hnm_idx", C.c_void_p), ("hnm", C.c_void_p)]


class _Aero(C.Structure):
    _fields_ = [("gamma", C.c_double), ("mach", C.c_double), ("reynolds", C.c_double),
                ("prandtl", C.c_double), ("tinf", C.c_double), ("twall", C.c_double),
                ("adiabatic", C.c_int)]


class _Report(C.Structure):
    _fields_ = [("tol", C.c_double), ("bnorm", C.c_double), ("n_est", C.c_int), ("est", C.c_void_p),
                ("gfinal", C.c_void_p), ("n_restarts_run", C.c_int), ("true_rel_res", C.c_double)]


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    """The restatement bound to one case (mesh + aero)."""

    def __init__(self, case):
        self.case = case
        nd = case.ndim
        self.ndim, self.nnod, self.neqn = nd, case.nnod, case.neqn
        self.Ke = self.nnod * self.neqn
        self._x = np.ascontiguousarray(case.nodes[:, :nd], dtype=np.float64)
        self._conn = np.ascontiguousarray(case.conn, dtype=np.int32)
        self._bc = np.ascontiguousarray(case.bc, dtype=np.int32)
        # adaptive elements: Hnm(N, M) stored at N + nnod*M, as the reference's Tensor
        adaptive = getattr(case, "adap_elements", None) is not None
        self._hidx = np.ascontiguousarray(case.hnm_index(), dtype=np.int32) if adaptive else None
        self._hnm = (np.ascontiguousarray(np.transpose(case.adap_hnm, (0, 2, 1)), dtype=np.float64)
                     if adaptive else None)
        self.mesh = _Mesh(nd, self.nnod, self.neqn, 2 if nd == 2 else 4, 4 if nd == 2 else 6,
                          case.n_nodes, case.n_elements, _p(self._x).value, _p(self._conn).value,
                          _p(self._bc).value, _p(self._hidx).value if adaptive else None,
                          _p(self._hnm).value if adaptive else None)
        a = case.aero
        self.aero = _Aero(float(a["gamma"]), float(a["M"]), float(a["Re"]), float(a["Pr"]), float(a["Tinf"]),
                          float(a["Twall"]), int(float(a["Adiabatic"])))
        self.L = lib()
        self.m = C.byref(self.mesh)
        self.a = C.byref(self.aero)

    @property
    def n_dof(self):
        return self.case.n_nodes * self.neqn

    def init_U(self):
        U = np.zeros(self.n_dof)
        prim = np.ascontiguousarray(self.case.nodes, dtype=np.float64)
        self.L.oracle_init_U(self.m, self.a, _p(prim), _p(U))
        return U

    def dirichlet(self):
        d = np.zeros(self.n_dof, dtype=np.uint8)
        self.L.oracle_dirichlet(self.m, self.a, _p(d))
        return d

    def rowmask(self):
        d = self.dirichlet()
        mk = np.zeros(self.case.n_elements, dtype=np.uint64)
        self.L.oracle_bc_rowmask(self.m, self.a, _p(d), _p(mk))
        return mk

    def cleng(self):
        c = np.zeros(self.case.n_elements)
        self.L.oracle_cleng(self.m, _p(c))
        return c

    def cfl(self, U, cfl, cleng=None):
        cleng = self.cleng() if cleng is None else cleng
        U = np.ascontiguousarray(U, dtype=np.float64)
        return self.L.oracle_cfl(self.m, self.a, _p(cleng), _p(U), float(cfl))

    def fdvparam(self, U):
        s = np.zeros((self.case.n_elements, 4))
        U = np.ascontiguousarray(U, dtype=np.float64)
        self.L.oracle_fdvparam(self.m, self.a, _p(U), _p(s))
        return s

    def form(self, U, dt, apply_bc=True, physical_3d_flux=False):
        """Element matrices, column-major per element: R[e, j, i] = R_e(i, j)."""
        E, Ke = self.case.n_elements, self.Ke
        R = np.zeros((E, Ke, Ke))
        rhs = np.zeros((E, Ke))
        U = np.ascontiguousarray(U, dtype=np.float64)
        self.L.oracle_form(self.m, self.a, _p(U), float(dt), int(apply_bc), int(physical_3d_flux), _p(R), _p(rhs))
        return R, rhs

    def compose_rhs(self, rhs):
        b = np.zeros(self.n_dof)
        self.L.oracle_compose_rhs(self.m, _p(np.ascontiguousarray(rhs)), _p(b))
        return b

    def matvec(self, R, x, transpose=False):
        y = np.zeros(self.n_dof)
        f = self.L.oracle_ebe_matvec_t if transpose else self.L.oracle_ebe_matvec
        f(self.m, _p(np.ascontiguousarray(R)), _p(np.ascontiguousarray(x, dtype=np.float64)), _p(y))
        return y

    def _report(self, cap_est, cap_fin):
        est = np.zeros(max(cap_est, 1))
        fin = np.zeros(max(cap_fin, 1))
        rep = _Report(0, 0, 0, _p(est).value, _p(fin).value, 0, 0)
        return rep, est, fin

    @staticmethod
    def _unpack(rep, est, fin):
        return {"tol": rep.tol, "bnorm": rep.bnorm, "est": est[: rep.n_est].copy(),
                "gfinal": fin[: rep.n_restarts_run].copy(), "restarts": rep.n_restarts_run,
                "true_rel_res": rep.true_rel_res}

    def gmres_ref(self, R, rhs, m, restart):
        du = np.zeros(self.n_dof)
        rep, est, fin = self._report(m * restart, restart)
        self.L.oracle_gmres_ref(self.m, _p(np.ascontiguousarray(R)), _p(np.ascontiguousarray(rhs)), int(m),
                                int(restart), _p(du), C.byref(rep))
        return du, self._unpack(rep, est, fin)

    def gmres_correct(self, R, rhs, m, max_restart, rtol):
        du = np.zeros(self.n_dof)
        rep, est, fin = self._report(m * max_restart, max_restart)
        self.L.oracle_gmres_correct(self.m, _p(np.ascontiguousarray(R)), _p(np.ascontiguousarray(rhs)), int(m),
                                    int(max_restart), float(rtol), _p(du), C.byref(rep))
        return du, self._unpack(rep, est, fin)

    def step(self, U, cfl, m, restart, mode=0, rtol=1e-8, physical_3d_flux=False, cleng=None):
        """One FDV step on a copy of U; returns (U_new, U0, dt, rms, report)."""
        cleng = self.cleng() if cleng is None else cleng
        U = np.array(U, dtype=np.float64, copy=True)
        U0 = np.zeros_like(U)
        dt = np.zeros(1)
        rms = np.zeros(self.neqn)
        rep, est, fin = self._report(m * restart, restart)
        self.L.oracle_step(self.m, self.a, _p(cleng), float(cfl), int(m), int(restart), int(mode), float(rtol),
                           int(physical_3d_flux), _p(U), _p(U0), _p(dt), _p(rms), C.byref(rep))
        return U, U0, float(dt[0]), rms, self._unpack(rep, est, fin)


def gauss(n=2):
    z = np.zeros(n)
    w = np.zeros(n)
    lib().oracle_gauss(int(n), _p(z), _p(w))
    return z, w


def read_records(path: str) -> dict:
    """Read a record file written by oracle/_ref/cfdv_ref into {name: ndarray}."""
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        n = int.from_bytes(data[pos:pos + 4], "little"); pos += 4
        name = data[pos:pos + n].decode(); pos += n
        t = chr(data[pos]); pos += 1
        cnt = int.from_bytes(data[pos:pos + 8], "little"); pos += 8
        dt = np.float64 if t == "d" else np.int32
        nb = cnt * (8 if t == "d" else 4)
        out[name] = np.frombuffer(data[pos:pos + nb], dtype=dt).copy()
        pos += nb
    return out


def run_reference(case_dir: str, out_path: str, steps: int = 1, dump_step: int = -1,
                  gmresiter: int | None = None, restart: int | None = None, extra=(),
                  timeout: float = 3600) -> dict:
    """Run the reference build on a case directory and return its records; `extra` holds
    further driver options (ref_driver.cpp: --elements FILE, --form-subset, --tecplot)."""
    if not os.path.exists(REF_BIN):
        raise FileNotFoundError(f"reference build missing: {REF_BIN}")
    cmd = [REF_BIN, case_dir, out_path, "--steps", str(steps), "--dump-step", str(dump_step), "--quiet"]
    if gmresiter:
        cmd += ["--gmresiter", str(gmresiter)]
    if restart:
        cmd += ["--restart", str(restart)]
    cmd += list(extra)
    # the reference stops at std::cin.get() on mesh errors (calc_TF_norm3D.h:137-144); give it no input
    subprocess.run(cmd, check=True, stdin=subprocess.DEVNULL, timeout=timeout)
    return read_records(out_path)
