"""ctypes binding of libcfdv_gpu.so (include/cfdv_gpu.h) for Python callers.

``FDVSolver`` mirrors the objects the reference driver owns per case
(src/main.cpp:104-197): the mesh and node state, the element matrices formed each
step, and the GMRES solver (``GMRESbase``, Utility/Solvers/GMRESbase.h:8-23).
There is no CPU implementation behind it: if the CUDA library is missing or no GPU
is present the constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcfdv_gpu.so")

PREC_FP64, PREC_MIXED = 0, 1
GMRES_REFERENCE, GMRES_CORRECT = 0, 1

STATUS = {0: "ok", 1: "bad argument", 2: "CUDA error", 3: "bad mesh", 4: "non-finite value",
          5: "allocation failed", 6: "call out of order", 7: "not converged",
          8: "size beyond the static scratch limit"}

# every entry point declared in include/cfdv_gpu.h
EXPORTS = ["cfdv_create", "cfdv_upload_mesh", "cfdv_destroy", "cfdv_last_error", "cfdv_get_stream",
           "cfdv_set_state", "cfdv_load_node_records", "cfdv_get_state", "cfdv_state_device_ptr", "cfdv_cfl",
           "cfdv_form", "cfdv_set_element_matrices", "cfdv_gmres", "cfdv_update", "cfdv_rms", "cfdv_step", "cfdv_get_fdv_params",
           "cfdv_get_element_matrices", "cfdv_get_rhs_vector", "cfdv_get_du", "cfdv_matvec", "cfdv_profile",
           "cfdv_profile_read", "cfdv_vjp", "cfdv_jvp", "cfdv_element_functional", "cfdv_wall_force",
           "cfdv_wall_nodes", "cfdv_adjoint", "cfdv_tangent", "cfdv_ebe_matvec_static", "cfdv_set_adaptive",
           "cfdv_step_host", "cfdv_get_element_subset", "cfdv_refine_marks"]


class CfdvError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cfdv error {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


class _Mesh(C.Structure):
    _fields_ = [("ndim", C.c_int), ("n_nodes", C.c_int), ("n_elements", C.c_int),
                ("x", C.c_void_p), ("conn", C.c_void_p), ("bc", C.c_void_p)]


class _Params(C.Structure):
    _fields_ = [("gamma", C.c_double), ("mach", C.c_double), ("reynolds", C.c_double), ("prandtl", C.c_double),
                ("tinf", C.c_double), ("twall", C.c_double), ("adiabatic", C.c_int), ("physical_3d_flux", C.c_int)]


class _Opts(C.Structure):
    _fields_ = [("mode", C.c_int), ("m", C.c_int), ("restarts", C.c_int), ("rtol", C.c_double),
                ("precision", C.c_int), ("true_residual", C.c_int), ("engine", C.c_int), ("precond", C.c_int),
                ("orth", C.c_int), ("warm_start", C.c_int)]


class _Report(C.Structure):
    _fields_ = [("tol", C.c_double), ("bnorm", C.c_double), ("n_est", C.c_int), ("est_capacity", C.c_int),
                ("est", C.c_void_p), ("gfinal_capacity", C.c_int), ("gfinal", C.c_void_p),
                ("n_restarts", C.c_int), ("n_matvec", C.c_int), ("true_rel_res", C.c_double)]


class _Stats(C.Structure):
    _fields_ = [("launches", C.c_long), ("total_ms", C.c_double), ("bytes", C.c_double),
                ("form_launches", C.c_long), ("form_ms", C.c_double), ("kernel_launches", C.c_long),
                ("solves", C.c_long), ("solve_ms", C.c_double), ("solve_bytes", C.c_double),
                ("matvec_ms", C.c_double), ("matvec_bytes", C.c_double)]


class _AdjOpts(C.Structure):
    _fields_ = [("n_steps", C.c_int), ("checkpoint_every", C.c_int), ("cfl", C.c_double), ("m", C.c_int),
                ("restarts", C.c_int), ("rtol", C.c_double), ("precision", C.c_int), ("wall_bc", C.c_int),
                ("max_kept_sets", C.c_int)]


class _AdjResult(C.Structure):
    _fields_ = [("J", C.c_double), ("dJ_dmach", C.c_double), ("dJ_dtwall", C.c_double), ("n_wall_nodes", C.c_int),
                ("wall_capacity", C.c_int), ("wall_nodes", C.c_void_p), ("dJ_dtnode", C.c_void_p),
                ("forward_ms", C.c_double), ("backward_ms", C.c_double), ("forward_matvecs", C.c_int),
                ("adjoint_matvecs", C.c_int), ("kept_matrix_sets", C.c_int), ("reverse_forms", C.c_int)]


_lib = None


def lib():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA library not built: {LIB_PATH} (run __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        P, I, D = C.c_void_p, C.c_int, C.c_double
        L.cfdv_create.argtypes = [P, P, P]
        L.cfdv_upload_mesh.argtypes = [P, P]
        L.cfdv_set_adaptive.argtypes = [P, C.c_int, P, P]
        L.cfdv_destroy.argtypes = [P]
        L.cfdv_destroy.restype = None
        L.cfdv_last_error.argtypes = [P]
        L.cfdv_last_error.restype = C.c_char_p
        L.cfdv_get_stream.argtypes = [P, P]
        L.cfdv_set_state.argtypes = [P, P, C.c_size_t]
        L.cfdv_load_node_records.argtypes = [P, P, C.c_size_t]
        L.cfdv_get_state.argtypes = [P, P, P, C.c_size_t]
        L.cfdv_state_device_ptr.argtypes = [P, P]
        L.cfdv_cfl.argtypes = [P, D, P]
        L.cfdv_form.argtypes = [P, D, I]
        L.cfdv_set_element_matrices.argtypes = [P, P, P, I]
        L.cfdv_gmres.argtypes = [P, P, P]
        L.cfdv_update.argtypes = [P]
        L.cfdv_rms.argtypes = [P, P]
        L.cfdv_step.argtypes = [P, D, P, P, P]
        L.cfdv_step_host.argtypes = [P, D, P, P, P, P, P]
        L.cfdv_get_fdv_params.argtypes = [P, P]
        L.cfdv_get_element_matrices.argtypes = [P, P, P]
        L.cfdv_get_element_subset.argtypes = [P, I, P, P, P, P]
        L.cfdv_refine_marks.argtypes = [P, D, P, I, P]
        L.cfdv_get_rhs_vector.argtypes = [P, P]
        L.cfdv_get_du.argtypes = [P, P]
        L.cfdv_matvec.argtypes = [P, P, P, I, I]
        L.cfdv_profile.argtypes = [P, I]
        L.cfdv_profile_read.argtypes = [P, P]
        L.cfdv_vjp.argtypes = [P, P, P, P, P, P]
        L.cfdv_jvp.argtypes = [P, P, P, D, D, P]
        L.cfdv_element_functional.argtypes = [P, P, P, P]
        L.cfdv_wall_force.argtypes = [P, I, P, P, P]
        L.cfdv_wall_nodes.argtypes = [P, I, P, I, P]
        L.cfdv_adjoint.argtypes = [P, P, P]
        L.cfdv_tangent.argtypes = [P, P, D, P, P, P]
        L.cfdv_ebe_matvec_static.argtypes = [I, I, I, P, P, P, P, P, P, I, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class FDVSolver:
    """One mesh + state on the current CUDA device."""

    def __init__(self, case, physical_3d_flux: bool = False):
        self.L = lib()
        self.case = case
        self.ndim = case.ndim
        self.nnod, self.neqn = case.nnod, case.neqn
        self.Ke = self.nnod * self.neqn
        self.n_nodes, self.n_elements = case.n_nodes, case.n_elements
        self.n_dof = self.n_nodes * self.neqn
        self._x = np.ascontiguousarray(case.nodes[:, : self.ndim], dtype=np.float64)
        self._conn = np.ascontiguousarray(case.conn, dtype=np.int32)
        self._bc = np.ascontiguousarray(case.bc, dtype=np.int32)
        mesh = _Mesh(self.ndim, self.n_nodes, self.n_elements, _p(self._x).value, _p(self._conn).value,
                     _p(self._bc).value)
        a = case.aero
        params = _Params(float(a["gamma"]), float(a["M"]), float(a["Re"]), float(a["Pr"]), float(a["Tinf"]),
                         float(a["Twall"]), int(float(a["Adiabatic"])), int(bool(physical_3d_flux)))
        self._ctx = C.c_void_p()
        rc = self.L.cfdv_create(C.byref(mesh), C.byref(params), C.byref(self._ctx))
        if rc:
            msg = self.L.cfdv_last_error(self._ctx).decode() if self._ctx else ""
            if self._ctx:
                self.L.cfdv_destroy(self._ctx)
                self._ctx = C.c_void_p()
            raise CfdvError(rc, msg)
        if getattr(case, "adap_elements", None) is not None:
            self.set_adaptive(case.adap_elements, case.adap_hnm)

    def set_adaptive(self, elements, hnm):
        """Adaptive elements and their hanging-node matrices hnm[k][N, M] (cfdv_set_adaptive);
        an empty list clears them."""
        el = np.ascontiguousarray(elements, dtype=np.int32)
        # Hnm(N, M) stored at N + nnod*M
        h = np.ascontiguousarray(np.transpose(np.asarray(hnm, dtype=np.float64).reshape(len(el), self.nnod, self.nnod),
                                              (0, 2, 1)))
        self._ck(self.L.cfdv_set_adaptive(self._ctx, len(el), _p(el) if len(el) else None, _p(h) if len(el) else None))

    def _ck(self, rc):
        if rc:
            raise CfdvError(rc, self.L.cfdv_last_error(self._ctx).decode())

    def close(self):
        if self._ctx:
            self.L.cfdv_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state --
    def load_node_records(self):
        rec = np.ascontiguousarray(self.case.nodes, dtype=np.float64)
        self._ck(self.L.cfdv_load_node_records(self._ctx, _p(rec), self.n_nodes))

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        self._ck(self.L.cfdv_set_state(self._ctx, _p(U), U.size))

    def get_state(self, U0=False):
        U = np.empty(self.n_dof)
        if U0:
            U0a = np.empty(self.n_dof)
            self._ck(self.L.cfdv_get_state(self._ctx, _p(U), _p(U0a), self.n_dof))
            return U, U0a
        self._ck(self.L.cfdv_get_state(self._ctx, _p(U), None, self.n_dof))
        return U

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        self._ck(self.L.cfdv_get_stream(self._ctx, C.byref(s)))
        return s.value or 0

    @property
    def state_ptr(self) -> int:
        p = C.c_void_p()
        self._ck(self.L.cfdv_state_device_ptr(self._ctx, C.byref(p)))
        return p.value

    # -- the step --
    def cfl(self, cfl: float) -> float:
        dt = C.c_double()
        self._ck(self.L.cfdv_cfl(self._ctx, float(cfl), C.byref(dt)))
        return dt.value

    def form(self, dt: float, precision: int = PREC_FP64):
        self._ck(self.L.cfdv_form(self._ctx, float(dt), int(precision)))

    def set_element_matrices(self, R, rhs, precision: int = PREC_FP64):
        R = np.ascontiguousarray(R, dtype=np.float64)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        assert R.size == self.n_elements * self.Ke * self.Ke and rhs.size == self.n_elements * self.Ke
        self._ck(self.L.cfdv_set_element_matrices(self._ctx, _p(R), _p(rhs), int(precision)))

    @staticmethod
    def _opts(mode, m, restarts, rtol, precision, true_residual, engine=0, precond=1, orth=2, warm_start=False):
        return _Opts(int(mode), int(m), int(restarts), float(rtol), int(precision), int(bool(true_residual)),
                     int(engine), int(precond), int(orth), int(bool(warm_start)))

    def _report(self, m, restarts):
        """Report struct and history buffers for (m, restarts), kept between calls (the
        returned dict copies what it needs)."""
        key = (m, restarts)
        cache = self.__dict__.setdefault("_rep_cache", {})
        if key not in cache:
            est = np.zeros(max(m * max(restarts, 1), 1))
            fin = np.zeros(max(restarts, 1))
            cache[key] = (_Report(0, 0, 0, est.size, _p(est).value, fin.size, _p(fin).value, 0, 0, -1.0), est, fin)
        rep, est, fin = cache[key]
        rep.tol = rep.bnorm = 0.0
        rep.n_est = rep.n_restarts = rep.n_matvec = 0
        rep.true_rel_res = -1.0
        return rep, est, fin

    @staticmethod
    def _unpack(rep, est, fin):
        return {"tol": rep.tol, "bnorm": rep.bnorm, "est": est[: min(rep.n_est, est.size)].copy(),
                "gfinal": fin[: min(rep.n_restarts, fin.size)].copy(), "restarts": rep.n_restarts,
                "matvecs": rep.n_matvec, "true_rel_res": rep.true_rel_res}

    def gmres(self, mode=GMRES_REFERENCE, m=20, restarts=1, rtol=1e-8, precision=PREC_FP64, true_residual=False,
              engine=0, precond=True, orth=2, warm_start=False):
        o = self._opts(mode, m, restarts, rtol, precision, true_residual, engine, precond, orth, warm_start)
        rep, est, fin = self._report(m, restarts)
        self._ck(self.L.cfdv_gmres(self._ctx, C.byref(o), C.byref(rep)))
        return self._unpack(rep, est, fin)

    def update(self):
        self._ck(self.L.cfdv_update(self._ctx))

    def rms(self):
        r = np.zeros(self.neqn)
        self._ck(self.L.cfdv_rms(self._ctx, _p(r)))
        return r

    def step(self, cfl, mode=GMRES_REFERENCE, m=20, restarts=1, rtol=1e-8, precision=PREC_FP64,
             true_residual=False, engine=0, precond=True, orth=2, warm_start=False):
        o = self._opts(mode, m, restarts, rtol, precision, true_residual, engine, precond, orth, warm_start)
        rep, est, fin = self._report(m, restarts)
        dt = C.c_double()
        self._ck(self.L.cfdv_step(self._ctx, float(cfl), C.byref(o), C.byref(rep), C.byref(dt)))
        out = self._unpack(rep, est, fin)
        out["dt"] = dt.value
        return out

    def step_host(self, cfl, U_in, U_out, mode=GMRES_REFERENCE, m=20, restarts=1, rtol=1e-8, precision=PREC_FP64,
                  true_residual=False, engine=0, precond=True, orth=2, warm_start=False):
        """step() with the state passed in and out as host float64 arrays (None: not copied);
        one host synchronisation for copies and step together."""
        for a in (U_in, U_out):
            if a is not None:
                assert a.dtype == np.float64 and a.size == self.n_dof and a.flags.c_contiguous
        o = self._opts(mode, m, restarts, rtol, precision, true_residual, engine, precond, orth, warm_start)
        rep, est, fin = self._report(m, restarts)
        dt = C.c_double()
        self._ck(self.L.cfdv_step_host(self._ctx, float(cfl), C.byref(o), C.byref(rep), C.byref(dt),
                                       None if U_in is None else _p(U_in), None if U_out is None else _p(U_out)))
        out = self._unpack(rep, est, fin)
        out["dt"] = dt.value
        return out

    # -- inspection --
    def fdv_params(self):
        s = np.zeros((self.n_elements, 4))
        self._ck(self.L.cfdv_get_fdv_params(self._ctx, _p(s)))
        return s

    def element_matrices(self):
        R = np.zeros((self.n_elements, self.Ke, self.Ke))
        rhs = np.zeros((self.n_elements, self.Ke))
        self._ck(self.L.cfdv_get_element_matrices(self._ctx, _p(R), _p(rhs)))
        return R, rhs

    def element_subset(self, ids):
        """(R [n, Ke, Ke] column-major per element as element_matrices(), rhs [n, Ke],
        s1..s4 [n, 4]) of the listed elements, copied alone."""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        R = np.zeros((ids.size, self.Ke, self.Ke))
        rhs = np.zeros((ids.size, self.Ke))
        s = np.zeros((ids.size, 4))
        self._ck(self.L.cfdv_get_element_subset(self._ctx, ids.size, _p(ids), _p(R), _p(rhs), _p(s)))
        return R, rhs, s

    def refine_marks(self, threshold=0.8):
        """Element ids with s1 > threshold at the current state (the reference's refinement
        criterion), ascending."""
        n = C.c_int()
        self._ck(self.L.cfdv_refine_marks(self._ctx, float(threshold), None, 0, C.byref(n)))
        ids = np.zeros(max(n.value, 1), dtype=np.int32)
        self._ck(self.L.cfdv_refine_marks(self._ctx, float(threshold), _p(ids), ids.size, C.byref(n)))
        return ids[: n.value].copy()

    def upload_case(self, case):
        """Replace the mesh by `case`'s (a refined mesh from the host): cfdv_upload_mesh, then
        the adaptive elements of `case` if it has any (cfdv_set_adaptive).  The state and the
        matrices are reset; load node records or set the state next."""
        ndim = case.ndim
        assert ndim == self.ndim
        self._x = np.ascontiguousarray(case.nodes[:, :ndim], dtype=np.float64)
        self._conn = np.ascontiguousarray(case.conn, dtype=np.int32)
        self._bc = np.ascontiguousarray(case.bc, dtype=np.int32)
        mesh = _Mesh(ndim, case.n_nodes, case.n_elements, _p(self._x).value, _p(self._conn).value, _p(self._bc).value)
        self._ck(self.L.cfdv_upload_mesh(self._ctx, C.byref(mesh)))
        self.case = case
        self.n_nodes, self.n_elements = case.n_nodes, case.n_elements
        self.n_dof = self.n_nodes * self.neqn
        self.__dict__.pop("_rep_cache", None)
        if getattr(case, "adap_elements", None) is not None:
            self.set_adaptive(case.adap_elements, case.adap_hnm)

    def rhs_vector(self):
        b = np.zeros(self.n_dof)
        self._ck(self.L.cfdv_get_rhs_vector(self._ctx, _p(b)))
        return b

    def du(self):
        d = np.zeros(self.n_dof)
        self._ck(self.L.cfdv_get_du(self._ctx, _p(d)))
        return d

    def matvec(self, x, precision=PREC_FP64, transpose=False):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.n_dof)
        self._ck(self.L.cfdv_matvec(self._ctx, _p(x), _p(y), int(precision), int(bool(transpose))))
        return y

    def profile(self, enable=True):
        self._ck(self.L.cfdv_profile(self._ctx, int(bool(enable))))

    def profile_read(self):
        s = _Stats()
        self._ck(self.L.cfdv_profile_read(self._ctx, C.byref(s)))
        return {"launches": s.launches, "total_ms": s.total_ms, "bytes": s.bytes,
                "form_launches": s.form_launches, "form_ms": s.form_ms,
                "kernel_launches": s.kernel_launches, "solves": s.solves, "solve_ms": s.solve_ms,
                "solve_bytes": s.solve_bytes, "matvec_ms": s.matvec_ms, "matvec_bytes": s.matvec_bytes}

    # -- discrete adjoint and tangent --
    def vjp(self, mu, du):
        """(dr/dU)^T mu assembled, mu^T dr/ddt, mu^T dr/dMach at the current U and formed dt."""
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        du = np.ascontiguousarray(du, dtype=np.float64)
        g = np.zeros(self.n_dof)
        gd, gm = C.c_double(), C.c_double()
        self._ck(self.L.cfdv_vjp(self._ctx, _p(mu), _p(du), _p(g), C.byref(gd), C.byref(gm)))
        return g, gd.value, gm.value

    def jvp(self, du, tU, t_dt=0.0, t_mach=0.0):
        du = np.ascontiguousarray(du, dtype=np.float64)
        tU = np.ascontiguousarray(tU, dtype=np.float64)
        dr = np.zeros(self.n_dof)
        self._ck(self.L.cfdv_jvp(self._ctx, _p(du), _p(tU), float(t_dt), float(t_mach), _p(dr)))
        return dr

    def element_functional(self, mu, du):
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        du = np.ascontiguousarray(du, dtype=np.float64)
        L = np.zeros(self.n_elements)
        self._ck(self.L.cfdv_element_functional(self._ctx, _p(mu), _p(du), _p(L)))
        return L

    def wall_force(self, wall_bc=1, grad=False):
        F = C.c_double()
        dm = C.c_double()
        g = np.zeros(self.n_dof) if grad else None
        self._ck(self.L.cfdv_wall_force(self._ctx, int(wall_bc), C.byref(F), _p(g) if grad else None,
                                        C.byref(dm)))
        return (F.value, g, dm.value) if grad else F.value

    def wall_nodes(self, wall_bc=1):
        n = C.c_int()
        self._ck(self.L.cfdv_wall_nodes(self._ctx, int(wall_bc), None, 0, C.byref(n)))
        ids = np.zeros(max(n.value, 1), dtype=np.int32)
        self._ck(self.L.cfdv_wall_nodes(self._ctx, int(wall_bc), _p(ids), ids.size, C.byref(n)))
        return ids[: n.value].copy()

    @staticmethod
    def _adj_opts(n_steps, checkpoint_every, cfl, m, restarts, rtol, precision, wall_bc, max_kept_sets=0):
        return _AdjOpts(int(n_steps), int(checkpoint_every), float(cfl), int(m), int(restarts), float(rtol),
                        int(precision), int(wall_bc), int(max_kept_sets))

    def adjoint(self, n_steps, cfl, checkpoint_every=50, m=30, restarts=200, rtol=1e-10, precision=PREC_FP64,
                wall_bc=1, max_kept_sets=0):
        """Gradient of J = mean_{n=1..N} F_x(U_n) w.r.t. Mach, wall temperature and each wall-node T0.
        max_kept_sets: element-matrix sets kept for the reverse steps (0: as many as fit, -1: none)."""
        o = self._adj_opts(n_steps, checkpoint_every, cfl, m, restarts, rtol, precision, wall_bc, max_kept_sets)
        nw = len(self.wall_nodes(wall_bc))
        ids = np.zeros(max(nw, 1), dtype=np.int32)
        gT = np.zeros(max(nw, 1))
        r = _AdjResult(0, 0, 0, 0, nw, _p(ids).value, _p(gT).value, 0, 0, 0, 0, 0, 0)
        self._ck(self.L.cfdv_adjoint(self._ctx, C.byref(o), C.byref(r)))
        return {"J": r.J, "dJ_dmach": r.dJ_dmach, "dJ_dtwall": r.dJ_dtwall, "wall_nodes": ids[:nw].copy(),
                "dJ_dtnode": gT[:nw].copy(), "forward_ms": r.forward_ms, "backward_ms": r.backward_ms,
                "forward_matvecs": r.forward_matvecs, "adjoint_matvecs": r.adjoint_matvecs,
                "kept_matrix_sets": r.kept_matrix_sets, "reverse_forms": r.reverse_forms}

    def tangent(self, n_steps, cfl, dmach=0.0, dT_wall=None, m=30, restarts=200, rtol=1e-10, precision=PREC_FP64,
                wall_bc=1):
        """FP64 tangent-linear run: (J, dJ) along (dmach, dT_wall per wall node)."""
        o = self._adj_opts(n_steps, 1, cfl, m, restarts, rtol, precision, wall_bc)
        J, dJ = C.c_double(), C.c_double()
        dT = None if dT_wall is None else np.ascontiguousarray(dT_wall, dtype=np.float64)
        self._ck(self.L.cfdv_tangent(self._ctx, C.byref(o), float(dmach), _p(dT) if dT is not None else None,
                                     C.byref(J), C.byref(dJ)))
        return J.value, dJ.value
