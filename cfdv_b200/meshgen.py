"""Synthetic FDV cases written in the CFDV reference's on-disk case format.

A case directory holds exactly what the reference driver loads:

* ``binarynodes``    packed float64 records ``{x[ndim], rho, v[ndim], T}``
                     (``node_2d_t``/``node_3d_t``, src/Utility/IO/ASCIItoBinary/LoadBinary.h:20-41)
* ``binaryelements`` packed int32 records ``{node[nnod], bc[nface]}``
                     (``ele_2d_t``/``ele_3d_t``, LoadBinary.h:28-47)
* ``control`` / ``aero``  ``key = value`` files with the keys registered at
                     src/MPIBinaryConfiguration.h:29-63
* ``MPIBreakdown``   the single-rank partition line (src/Utility/MPI_Breakdown.h:23-70)

Element-local node order follows the reference: quad4 counter-clockwise,
hex8 nodes 0-3 the bottom (zeta=-1) counter-clockwise and 4-7 above them.
Face ``f`` of a quad is the edge (f, f+1 mod 4) (src/FiniteElement/get_face.h:80-89);
hex faces are 0:(3,2,1,0) zeta=-1, 1:(0,1,5,4) eta=-1, 2:(1,2,6,5) xi=+1,
3:(2,3,7,6) eta=+1, 4:(3,0,4,7) xi=-1, 5:(6,7,4,5) zeta=+1 (get_face.h:106-164).
Boundary codes follow the reference's examples: -1 inflow (all DOFs fixed),
1/11/21/31 no-slip walls, 2/22 symmetry, 4 ramp wall, 6 outflow, 7 top, 8 ramp exit.

Random perturbations use ``numpy.random.default_rng(SEED)`` with ``SEED = 20261203``.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

SEED = 20261203


@dataclass
class Case:
    name: str
    ndim: int
    nodes: np.ndarray  # (Nn, 2*ndim+2) float64: x[ndim], rho, v[ndim], T
    elements: np.ndarray  # (E, nnod+nface) int32: node ids then bc codes
    control: dict = field(default_factory=dict)
    aero: dict = field(default_factory=dict)
    # adaptive (hanging-node) elements: ids, refine levels and Hnm[N, M] (nnod x nnod), as the
    # reference's "adap" file holds them (LoadBinary.h:247-261, Element.h:39-40)
    adap_elements: np.ndarray | None = None
    adap_levels: np.ndarray | None = None
    adap_hnm: np.ndarray | None = None

    @property
    def nnod(self) -> int:
        return 4 if self.ndim == 2 else 8

    @property
    def nface(self) -> int:
        return 4 if self.ndim == 2 else 6

    @property
    def neqn(self) -> int:
        return self.ndim + 2

    @property
    def n_nodes(self) -> int:
        return self.nodes.shape[0]

    @property
    def n_elements(self) -> int:
        return self.elements.shape[0]

    @property
    def conn(self) -> np.ndarray:
        return self.elements[:, : self.nnod]

    @property
    def bc(self) -> np.ndarray:
        return self.elements[:, self.nnod:]

    def hnm_index(self) -> np.ndarray:
        """Per element the row of ``adap_hnm`` that applies, -1 for a plain element."""
        idx = np.full(self.n_elements, -1, dtype=np.int32)
        if self.adap_elements is not None:
            idx[self.adap_elements] = np.arange(len(self.adap_elements), dtype=np.int32)
        return idx


def _control(ndim, Nn, E, cfl, m, restart=1, itermax=1000):
    return {
        "itermax": itermax, "cfl": cfl, "gmresrestart": restart, "gmresiter": m,
        "ndim": ndim, "nnod": 4 if ndim == 2 else 8, "neqn": ndim + 2,
        "nbnod": 2 if ndim == 2 else 4, "nface": 4 if ndim == 2 else 6,
        "nodes": Nn, "elements": E, "iter": 0, "adap": 0,
    }


def _aero(M, Re, adiabatic, Twall, Pr=0.72, Tinf=216.6666, gamma=1.4):
    return {"M": M, "Pr": Pr, "Re": Re, "Tinf": Tinf, "Twall": Twall,
            "Adiabatic": int(bool(adiabatic)), "gamma": gamma}


def _quad_grid(X, Y):
    """Structured (nx+1)x(ny+1) node grid -> node coords and CCW quad connectivity.
    Node id = j*(nx+1)+i; element id = j*nx+i."""
    ny1, nx1 = X.shape
    nx, ny = nx1 - 1, ny1 - 1
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny))
    n0 = (jj * nx1 + ii).ravel()
    conn = np.stack([n0, n0 + 1, n0 + 1 + nx1, n0 + nx1], axis=1).astype(np.int32)
    xy = np.stack([X.ravel(), Y.ravel()], axis=1)
    return xy, conn, ii.ravel(), jj.ravel()


def _hex_grid(X, Y, Z, periodic_i=False, periodic_j=False):
    """Structured hex grid from node arrays shaped (nk, nj, ni) (k = zeta direction).
    Node id = (k*nj + j)*ni + i.  With periodic_i / periodic_j the last element layer
    connects back to index 0 (the arrays then hold ni / nj distinct node layers)."""
    nk, nj, ni = X.shape
    ne_i = ni if periodic_i else ni - 1
    ne_j = nj if periodic_j else nj - 1
    ne_k = nk - 1
    kk, jj, ii = np.meshgrid(np.arange(ne_k), np.arange(ne_j), np.arange(ne_i), indexing="ij")
    i1 = (ii + 1) % ni
    j1 = (jj + 1) % nj

    def nid(k, j, i):
        return (k * nj + j) * ni + i

    conn = np.stack([
        nid(kk, jj, ii), nid(kk, jj, i1), nid(kk, j1, i1), nid(kk, j1, ii),
        nid(kk + 1, jj, ii), nid(kk + 1, jj, i1), nid(kk + 1, j1, i1), nid(kk + 1, j1, ii),
    ], axis=-1).reshape(-1, 8).astype(np.int32)
    xyz = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    return xyz, conn, ii.ravel(), jj.ravel(), kk.ravel(), (ne_i, ne_j, ne_k)


def _pack(ndim, x, rho, v, T):
    Nn = x.shape[0]
    out = np.zeros((Nn, 2 * ndim + 2), dtype=np.float64)
    out[:, :ndim] = x
    out[:, ndim] = rho
    out[:, ndim + 1: 2 * ndim + 1] = v
    out[:, 2 * ndim + 1] = T
    return out


def lid(n: int = 32, M: float = 0.1, Re: float = 100.0, cfl: float = 0.5, m: int = 20,
        steps: int = 200) -> Case:
    """Lid-driven cavity: uniform n x n quad4 on [0,1]^2, lid (top, bc -1) moving at u=1
    (lid Mach = M), isothermal no-slip walls (bc 1, Adiabatic = 0), fluid at rest with
    rho = 1, T = 1.  Lid corner nodes keep u = 0 as in the reference's Lid examples."""
    s = np.linspace(0.0, 1.0, n + 1)
    X, Y = np.meshgrid(s, s)
    xy, conn, ii, jj = _quad_grid(X, Y)
    Nn = xy.shape[0]
    v = np.zeros((Nn, 2))
    top = np.isclose(xy[:, 1], 1.0) & (xy[:, 0] > 0) & (xy[:, 0] < 1)
    v[top, 0] = 1.0
    nodes = _pack(2, xy, np.ones(Nn), v, np.ones(Nn))
    bc = np.zeros((conn.shape[0], 4), dtype=np.int32)
    bc[jj == 0, 0] = 1
    bc[ii == n - 1, 1] = 1
    bc[jj == n - 1, 2] = -1
    bc[ii == 0, 3] = 1
    el = np.concatenate([conn, bc], axis=1)
    return Case(f"lid{n}", 2, nodes, el, _control(2, Nn, el.shape[0], cfl, m, itermax=steps),
                _aero(M, Re, adiabatic=False, Twall=1.0))


def plate(nx: int = 200, ny: int = 100, M: float = 3.0, Re: float = 1.0e4, cfl: float = 1.0,
          m: int = 30, steps: int = 2000, ratio: float = 1.05, noise: float = 1e-3) -> Case:
    """Supersonic flat plate: x in [0, 1.1] with the adiabatic plate (bc 1) from x = 0.1 and
    symmetry (bc 2) ahead of it, inflow -1, top 7, outflow 6; y in [0, 0.75] stretched
    geometrically (ratio 1.05).  Freestream rho = 1, u = 1, T = 1 with seeded 1e-3 relative
    Gaussian noise on rho at interior nodes.  Over the plate the start is a smooth
    boundary-layer profile u = tanh(y / 0.005), T = Tr + (1 - Tr) u^2 (Tr the recovery
    temperature), wall nodes at rest: with an exact linear solve, an impulsive start (wall
    at rest next to freestream across the 3e-4 first cell) drives the density negative in
    the first step."""
    n_lead = max(1, int(round(nx * 0.1 / 1.1)))
    xs = np.concatenate([np.linspace(0.0, 0.1, n_lead + 1)[:-1], np.linspace(0.1, 1.1, nx - n_lead + 1)])
    dy = np.array([ratio ** k for k in range(ny)])
    ys = np.concatenate([[0.0], np.cumsum(dy)]) * (0.75 / dy.sum())
    X, Y = np.meshgrid(xs, ys)
    xy, conn, ii, jj = _quad_grid(X, Y)
    Nn = xy.shape[0]
    gamma = 1.4
    Trec = 1.0 + 0.5 * (gamma - 1.0) * M * M
    rho = np.ones(Nn)
    v = np.zeros((Nn, 2))
    v[:, 0] = 1.0
    T = np.ones(Nn)
    onplate = xy[:, 0] >= 0.1 - 1e-12
    prof = np.tanh(xy[:, 1] / 0.005)
    v[onplate, 0] = prof[onplate]
    T[onplate] = Trec + (1.0 - Trec) * prof[onplate] ** 2
    interior = (xy[:, 0] > 0) & (xy[:, 0] < 1.1 - 1e-12) & (xy[:, 1] > 0) & (xy[:, 1] < 0.75 - 1e-12)
    rng = np.random.default_rng(SEED)
    rho[interior] *= 1.0 + noise * rng.standard_normal(int(interior.sum()))
    nodes = _pack(2, xy, rho, v, T)
    bc = np.zeros((conn.shape[0], 4), dtype=np.int32)
    xleft = xs[ii]
    bc[(jj == 0) & (xleft >= 0.1 - 1e-12), 0] = 1
    bc[(jj == 0) & (xleft < 0.1 - 1e-12), 0] = 2
    bc[ii == nx - 1, 1] = 6
    bc[jj == ny - 1, 2] = 7
    bc[ii == 0, 3] = -1
    el = np.concatenate([conn, bc], axis=1)
    return Case(f"plate{nx}x{ny}", 2, nodes, el, _control(2, Nn, el.shape[0], cfl, m, itermax=steps),
                _aero(M, Re, adiabatic=True, Twall=Trec))


def ramp(nx: int = 128, nz: int = 64, ny: int = 32, M: float = 2.5, Re: float = 1.0e5,
         Tw: float = 2.5, cfl: float = 0.25, m: int = 50, steps: int = 500,
         angle_deg: float = 15.0) -> Case:
    """3D compression ramp (x streamwise in [0,1], z wall-normal to 0.5, y spanwise in [0,0.25]):
    flat no-slip wall (bc 1) up to the corner at x = 0.5, then a 15 degree ramp wall (bc 4);
    inflow -1 (xi=-1), ramp exit 8 (xi=+1), top symmetry 2 (zeta=+1), side wall 21 (y=0) and
    side symmetry 22 (y=max).  Isothermal walls: Adiabatic = 0, wall nodes at T = Tw, at rest."""
    L, xc, H, W = 1.0, 0.5, 0.5, 0.25
    xs = np.linspace(0.0, L, nx + 1)
    ys = np.linspace(0.0, W, ny + 1)
    zeta = np.linspace(0.0, 1.0, nz + 1)
    floor = np.where(xs > xc, (xs - xc) * math.tan(math.radians(angle_deg)), 0.0)
    Zk, Yk, Xk = np.meshgrid(zeta, ys, xs, indexing="ij")
    Fk = np.broadcast_to(floor[None, None, :], Xk.shape)
    Z = Fk + Zk * (H - Fk)
    xyz, conn, ii, jj, kk, (ne_i, ne_j, ne_k) = _hex_grid(Xk, Yk, Z)
    Nn = xyz.shape[0]
    rho = np.ones(Nn)
    v = np.zeros((Nn, 3))
    v[:, 0] = 1.0
    T = np.ones(Nn)
    bc = np.zeros((conn.shape[0], 6), dtype=np.int32)
    xl = xs[ii]
    bc[(kk == 0) & (xl < xc - 1e-12), 0] = 1
    bc[(kk == 0) & (xl >= xc - 1e-12), 0] = 4
    bc[jj == 0, 1] = 21
    bc[ii == ne_i - 1, 2] = 8
    bc[jj == ne_j - 1, 3] = 22
    bc[ii == 0, 4] = -1
    bc[kk == ne_k - 1, 5] = 2
    wall_nodes = np.zeros(Nn, dtype=bool)
    for f, code in ((0, None), (1, 21)):
        sel = bc[:, f] != 0
        faces = {0: [3, 2, 1, 0], 1: [0, 1, 5, 4]}[f]
        wall_nodes[np.unique(conn[sel][:, faces])] = True
    wall_nodes &= xyz[:, 0] > 1e-12
    v[wall_nodes] = 0.0
    T[wall_nodes] = Tw
    nodes = _pack(3, xyz, rho, v, T)
    el = np.concatenate([conn, bc], axis=1)
    return Case(f"ramp{nx}x{nz}x{ny}", 3, nodes, el, _control(3, Nn, el.shape[0], cfl, m, itermax=steps),
                _aero(M, Re, adiabatic=False, Twall=Tw))


def cylinder(nr: int = 96, nth: int = 128, nz: int = 16, M: float = 0.3, Re: float = 150.0,
             Tw: float = 1.0, cfl: float = 0.5, m: int = 40, steps: int = 1000,
             r0: float = 0.5, r1: float = 20.0, span: float = 2.0) -> Case:
    """Circular cylinder on a hex8 O-grid: local xi = theta (periodic by connectivity),
    eta = z (nz node layers, symmetry planes bc 2 at both span ends), zeta = r (geometric
    from r0 to r1).  The span is not periodic by connectivity: elements take their geometry
    from absolute node coordinates, so a wrapped z layer would be an inverted element.
    Wall (zeta=-1 face) is an isothermal no-slip wall (bc 1, Adiabatic = 0) whose nth*nz
    nodes are at rest at T = Tw; the outer face is inflow -1 on the upstream half (x < 0)
    and outflow 6 downstream.  Freestream rho = 1, u = 1, T = 1."""
    q = (r1 / r0) ** (1.0 / nr)
    rs = r0 * q ** np.arange(nr + 1)
    th = 2.0 * math.pi * np.arange(nth) / nth
    zs = np.linspace(0.0, span, nz)
    Rk, Zj, Ti = np.meshgrid(rs, zs, th, indexing="ij")
    X = Rk * np.cos(Ti)
    Y = Rk * np.sin(Ti)
    xyz, conn, ii, jj, kk, (ne_i, ne_j, ne_k) = _hex_grid(X, Y, Zj, periodic_i=True)
    Nn = xyz.shape[0]
    rho = np.ones(Nn)
    v = np.zeros((Nn, 3))
    v[:, 0] = 1.0
    T = np.ones(Nn)
    wall = np.isclose(np.hypot(xyz[:, 0], xyz[:, 1]), r0)
    v[wall] = 0.0
    T[wall] = Tw
    nodes = _pack(3, xyz, rho, v, T)
    bc = np.zeros((conn.shape[0], 6), dtype=np.int32)
    bc[kk == 0, 0] = 1
    bc[jj == 0, 1] = 2
    bc[jj == ne_j - 1, 3] = 2
    outer = kk == ne_k - 1
    thc = 2.0 * math.pi * (ii + 0.5) / nth
    bc[outer & (np.cos(thc) < 0), 5] = -1
    bc[outer & (np.cos(thc) >= 0), 5] = 6
    el = np.concatenate([conn, bc], axis=1)
    return Case(f"cylinder{nr}x{nth}x{nz}", 3, nodes, el, _control(3, Nn, el.shape[0], cfl, m, itermax=steps),
                _aero(M, Re, adiabatic=False, Twall=Tw))


def duct(nx: int = 200, ny: int = 100, nz: int = 50, M: float = 0.8, Re: float = 5.0e4,
         cfl: float = 0.5, m: int = 40, steps: int = 100, jitter: float = 0.1) -> Case:
    """Rectangular duct, x in [0,4] streamwise, y in [0,2], z in [0,1]; interior nodes jittered
    by seeded uniform +-10% of the local spacing.  No-slip adiabatic walls: z-planes bc 1,
    y=0 bc 21, y=max bc 31; inflow -1 at x=0, outflow 6 at x=max.  Freestream rho=1, u=1,
    T=1 in the interior, wall nodes at rest."""
    xs = np.linspace(0.0, 4.0, nx + 1)
    ys = np.linspace(0.0, 2.0, ny + 1)
    zs = np.linspace(0.0, 1.0, nz + 1)
    Zk, Yj, Xi = np.meshgrid(zs, ys, xs, indexing="ij")
    rng = np.random.default_rng(SEED)
    inner = np.zeros(Xi.shape, dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    n_in = int(inner.sum())
    d = rng.uniform(-jitter, jitter, size=(3, n_in))
    Xi = Xi.copy(); Yj = Yj.copy(); Zk = Zk.copy()
    Xi[inner] += d[0] * (xs[1] - xs[0])
    Yj[inner] += d[1] * (ys[1] - ys[0])
    Zk[inner] += d[2] * (zs[1] - zs[0])
    xyz, conn, ii, jj, kk, (ne_i, ne_j, ne_k) = _hex_grid(Xi, Yj, Zk)
    Nn = xyz.shape[0]
    rho = np.ones(Nn)
    v = np.zeros((Nn, 3))
    v[:, 0] = 1.0
    T = np.ones(Nn)
    wall = ((np.isclose(xyz[:, 2], 0) | np.isclose(xyz[:, 2], 1.0) | np.isclose(xyz[:, 1], 0)
             | np.isclose(xyz[:, 1], 2.0)) & (xyz[:, 0] > 1e-12))
    v[wall] = 0.0
    nodes = _pack(3, xyz, rho, v, T)
    bc = np.zeros((conn.shape[0], 6), dtype=np.int32)
    bc[kk == 0, 0] = 1
    bc[kk == ne_k - 1, 5] = 1
    bc[jj == 0, 1] = 21
    bc[jj == ne_j - 1, 3] = 31
    bc[ii == 0, 4] = -1
    bc[ii == ne_i - 1, 2] = 6
    el = np.concatenate([conn, bc], axis=1)
    return Case(f"duct{nx}x{ny}x{nz}", 3, nodes, el, _control(3, Nn, el.shape[0], cfl, m, itermax=steps),
                _aero(M, Re, adiabatic=True, Twall=1.0))


# The five workloads (full sizes) and small versions of each used by the parity tests.
FULL = {
    "lid": lambda: lid(32),
    "plate": lambda: plate(200, 100),
    "ramp": lambda: ramp(128, 64, 32),
    "cylinder": lambda: cylinder(96, 128, 16),
    "duct": lambda: duct(200, 100, 50),
}
SMALL = {
    "lid8": lambda: lid(8),
    "lid32": lambda: lid(32),
    "plate20": lambda: plate(20, 10),
    "ramp4": lambda: ramp(8, 4, 4),
    "cyl4": lambda: cylinder(6, 8, 4),
    "duct4": lambda: duct(8, 4, 4),
}


def with_adaptive(case: Case, elements, hnm, levels=None) -> Case:
    """A copy of ``case`` whose ``elements`` carry the hanging-node matrices ``hnm``
    ((n, nnod, nnod), Hnm[N, M]); written with control adap = 1 and an "adap" file."""
    import copy
    c = copy.copy(case)
    c.control = dict(case.control)
    c.control["adap"] = 1
    c.adap_elements = np.asarray(elements, dtype=np.int32)
    c.adap_hnm = np.asarray(hnm, dtype=np.float64).reshape(len(c.adap_elements), case.nnod, case.nnod)
    c.adap_levels = np.ones(len(c.adap_elements), dtype=np.int32) if levels is None else np.asarray(levels, np.int32)
    c.name = case.name + "_adap"
    return c


def adaptive_demo(case: Case) -> Case:
    """Every third element of ``case`` (boundary elements included) made adaptive with a
    hanging-node style Hnm: the identity with one or two local nodes moved to the midpoint
    of an edge they share with a neighbour, or a quarter of the way along it (rows of Hnm
    sum to one, so the shape functions keep the partition of unity and the element stays
    valid).  Entries are exact in six significant digits, the precision at which the
    reference writes and reads them."""
    nnod = case.nnod
    edges = [(0, 1), (1, 2), (2, 3), (3, 0)] if case.ndim == 2 else [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6)]
    els, hs = [], []
    for k, e in enumerate(range(0, case.n_elements, 3)):
        H = np.eye(nnod)
        a, b = edges[k % len(edges)]
        H[a, a], H[a, b] = 0.5, 0.5  # local node a at the midpoint of edge a-b
        if k % 2:
            c, d = edges[(k + 2) % len(edges)]
            if c not in (a, b):
                H[c] = 0.0
                H[c, c], H[c, d] = 0.75, 0.25
        els.append(e)
        hs.append(H)
    return with_adaptive(case, els, hs)


def write_case(case: Case, path: str) -> str:
    """Write ``case`` as a reference case directory at ``path`` (created if needed)."""
    os.makedirs(path, exist_ok=True)
    case.nodes.astype("<f8").tofile(os.path.join(path, "binarynodes"))
    case.elements.astype("<i4").tofile(os.path.join(path, "binaryelements"))
    with open(os.path.join(path, "control"), "w") as f:
        for k, v in case.control.items():
            f.write(f"{k} = {v}\n")
    if case.adap_elements is not None:
        # "elno adap refine_level" then the Tensor serialisation (TensorStream.h:95-145): type,
        # ndim, extents, the storage in index order N + nnod*M
        nnod = case.nnod
        with open(os.path.join(path, "adap"), "w") as f:
            for e, lev, H in zip(case.adap_elements, case.adap_levels, case.adap_hnm):
                vals = " ".join(repr(float(v)) for v in H.T.ravel())
                f.write(f"{int(e)} 1 {int(lev)} double 2 {nnod} {nnod} {vals}\n")
    with open(os.path.join(path, "aero"), "w") as f:
        for k, v in case.aero.items():
            f.write(f"{k} = {v}\n")
    with open(os.path.join(path, "MPIBreakdown"), "w") as f:
        f.write("1\nelemin, elemax, nodemin, nodemax, nedgenode_l, nedgenode_r, NodeIteratorMin, NodeIteratorMax\n")
        f.write(f"0 {case.n_elements} 0 {case.n_nodes - 1} 0 0 0 {case.n_nodes - 1}\n")
    return path


# local node order of each face (FiniteElement/get_face.h:80-89, 106-164)
_FACE2 = [[0, 1], [1, 2], [2, 3], [3, 0]]
_FACE3 = [[3, 2, 1, 0], [0, 1, 5, 4], [1, 2, 6, 5], [2, 3, 7, 6], [3, 0, 4, 7], [6, 7, 4, 5]]


def write_ascii_case(case: Case, path: str, U: np.ndarray) -> str:
    """Write ``case`` as the reference's ASCII case directory (the input of its CONVERT tool,
    AsciiLoad.h): control, aero, nodes "number x[ndim] U[ndim+2]" with the conserved state U
    (1-based numbers), elements "number node[nnod]" (1-based), faces "element face bc
    node[nbnod]" (0-based element, local face nodes) and the adap file if any."""
    os.makedirs(path, exist_ok=True)
    nd, ne = case.ndim, case.neqn
    Ur = np.asarray(U, dtype=np.float64).reshape(case.n_nodes, ne)
    with open(os.path.join(path, "control"), "w") as f:
        for k, v in case.control.items():
            f.write(f"{k} = {v}\n")
    with open(os.path.join(path, "aero"), "w") as f:
        for k, v in case.aero.items():
            f.write(f"{k} = {v}\n")
    with open(os.path.join(path, "nodes"), "w") as f:
        for n in range(case.n_nodes):
            vals = list(case.nodes[n, :nd]) + list(Ur[n])
            f.write(f"{n + 1} " + " ".join(repr(float(v)) for v in vals) + "\n")
    with open(os.path.join(path, "elements"), "w") as f:
        for e in range(case.n_elements):
            f.write(f"{e + 1} " + " ".join(str(int(v) + 1) for v in case.conn[e]) + "\n")
    faces = _FACE2 if nd == 2 else _FACE3
    with open(os.path.join(path, "faces"), "w") as f:
        for e in range(case.n_elements):
            for k, code in enumerate(case.bc[e]):
                if code != 0:
                    f.write(f"{e} {k} {int(code)} " + " ".join(str(v) for v in faces[k]) + "\n")
    if case.adap_elements is not None:
        nnod = case.nnod
        with open(os.path.join(path, "adap"), "w") as f:
            for e, lev, H in zip(case.adap_elements, case.adap_levels, case.adap_hnm):
                f.write(f"{int(e)} 1 {int(lev)} double 2 {nnod} {nnod} " +
                        " ".join(repr(float(v)) for v in H.T.ravel()) + "\n")
    return path


def _parse_kv(path):
    kv = {}
    with open(path) as f:
        for line in f:
            line = line.split("!")[0].split("#")[0]
            if "=" in line:
                k, v = line.split("=", 1)
                kv[k.strip()] = v.strip()
    return kv


def read_case(path: str) -> Case:
    """Load a reference case directory (binary mesh + control + aero)."""
    control = _parse_kv(os.path.join(path, "control"))
    aero = _parse_kv(os.path.join(path, "aero"))
    ndim = int(control["ndim"])
    nnod = int(control["nnod"])
    nface = 4 if ndim == 2 else 6
    Nn = int(control["nodes"])
    E = int(control["elements"])
    nodes = np.fromfile(os.path.join(path, "binarynodes"), dtype="<f8").reshape(-1, 2 * ndim + 2)[:Nn]
    el = np.fromfile(os.path.join(path, "binaryelements"), dtype="<i4").reshape(-1, nnod + nface)[:E]
    case = Case(os.path.basename(os.path.normpath(path)), ndim, np.ascontiguousarray(nodes),
                np.ascontiguousarray(el), control, aero)
    adap = os.path.join(path, "adap")
    if control.get("adap", "0").strip().lower() in ("1", "true") and os.path.exists(adap):
        els, levs, hs = [], [], []
        with open(adap) as f:
            for line in f:
                t = line.split()
                if not t:
                    continue
                ni, nj = int(t[5]), int(t[6])
                vals = np.array([float(v) for v in t[7:7 + ni * nj]])
                if int(t[1]) == 0:
                    continue
                els.append(int(t[0]))
                levs.append(int(t[2]))
                hs.append(vals.reshape(nj, ni).T)  # storage N + ni*M -> H[N, M]
        if els:
            case.adap_elements = np.array(els, dtype=np.int32)
            case.adap_levels = np.array(levs, dtype=np.int32)
            case.adap_hnm = np.array(hs)
    return case
