"""CUDA path against the reference build on the full-size synthetic configurations.

The fixtures (tests/golden/make_golden_full.py) hold what the CFDV reference sources,
compiled unmodified (oracle/_ref/cfdv_ref), computed on the meshes of
cfdv_b200.meshgen.FULL; the meshes are regenerated here from their seeded generators and
checked against the fixture's digest first.

  plate 200x100 quad4 (M 3, Re 1e4, CFL 1): 25 steps of the reference's own solver
        (GMRES(30), one restart, its stopping rule and back substitution) -- dt, the
        tolerance, every Givens estimate, g(m), RMS and U after every step;
  ramp 128x64x32 hex8 (262,144 elements): the same for 2 steps of GMRES(50);
  cylinder 96x128x16 and duct 200x100x50 (10^6 elements): step 0 -- dt over the whole
        mesh, and R, rhs after ApplyBC and s1..s4 of the sampled elements.

Every one of them also checks step 0's element matrices on the sampled elements (first and
last element of each pattern of face boundary codes, plus interior elements).

Bars, as for the small cases: element matrices <= 1e-12 of each element's largest entry,
rhs <= 1e-12 of the sample's largest entry, s1..s4 <= 1e-14; the reference-mode solve
<= 1e-10 in the estimate history, g(m) (on the history's scale) and U (on its largest
entry), and 1e-7 in the RMS line."""
import numpy as np
import pytest

from conftest import GOLDEN, elem_rel_err, rel_err

pytestmark = pytest.mark.gpu

import os  # noqa: E402

from cfdv_b200 import meshgen as mg  # noqa: E402

_cases = {}


def full_case(name):
    if name not in _cases:
        _cases.clear()  # one full-size mesh at a time
        _cases[name] = mg.FULL[name]()
    return _cases[name]


def fixture(name):
    case = full_case(name)
    g = dict(np.load(os.path.join(GOLDEN, f"{case.name}.npz")))
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_golden import case_digest
    assert str(g["digest"]) == case_digest(case), "mesh generator changed since the fixture was made"
    return case, g


@pytest.fixture(scope="module")
def G():
    from cfdv_b200 import gpu
    return gpu


def check_step0_formation(G, s, case, g):
    dt = s.cfl(float(case.control["cfl"]))
    assert dt == pytest.approx(float(g["dt_dump"][0]), rel=1e-12)
    s.form(dt)
    R, rhs, sp = s.element_subset(g["elements"])
    assert elem_rel_err(R, g["R_bc"]) <= 1e-12
    assert rel_err(rhs, g["rhs_bc"]) <= 1e-12
    assert rel_err(sp, g["s1234"]) <= 1e-14
    return dt


@pytest.mark.parametrize("name", ["cylinder", "duct"])
def test_step0_formation_full_size(G, name):
    case, g = fixture(name)
    with G.FDVSolver(case) as s:
        s.load_node_records()
        check_step0_formation(G, s, case, g)


def field_sums(U, neqn):
    u = U.reshape(-1, neqn)
    return np.concatenate([u.sum(axis=0), (u * u).sum(axis=0)])


@pytest.mark.parametrize("name", ["plate", "ramp"])
def test_reference_mode_steps_full_size(G, name):
    case, g = fixture(name)
    m, r, cfl = int(case.control["gmresiter"]), int(case.control["gmresrestart"]), float(case.control["cfl"])
    dofs = g["dof_sample"]
    with G.FDVSolver(case) as s:
        s.load_node_records()
        check_step0_formation(G, s, case, g)
        worst = {"est": 0.0, "gfinal": 0.0, "U": 0.0, "Usum": 0.0, "rms": 0.0}
        for k in range(int(g["steps"])):
            rep = s.step(cfl, mode=G.GMRES_REFERENCE, m=m, restarts=r)
            assert rep["dt"] == pytest.approx(g[f"dt@{k}"][0], rel=1e-12)
            assert rep["tol"] == pytest.approx(g[f"tol@{k}"][0], rel=1e-12)
            assert len(rep["est"]) == len(g[f"est@{k}"]), f"step {k}: iteration count"
            worst["est"] = max(worst["est"], rel_err(rep["est"], g[f"est@{k}"]))
            scale = np.abs(g[f"est@{k}"]).max()
            worst["gfinal"] = max(worst["gfinal"], float(np.abs(rep["gfinal"] - g[f"gfinal@{k}"]).max() / scale))
            U = s.get_state()
            worst["U"] = max(worst["U"], rel_err(U[dofs], g[f"Usample@{k}"]))
            worst["Usum"] = max(worst["Usum"], rel_err(field_sums(U, case.neqn), g[f"Usum@{k}"]))
            worst["rms"] = max(worst["rms"], rel_err(s.rms(), g[f"rms@{k}"]))
        last = int(g["steps"]) - 1
        if f"U@{last}" in g:
            worst["U"] = max(worst["U"], rel_err(U, g[f"U@{last}"]))
    print(name, worst)
    assert worst["est"] <= 1e-10
    assert worst["gfinal"] <= 1e-10
    assert worst["U"] <= 1e-10
    assert worst["Usum"] <= 1e-10
    assert worst["rms"] <= 1e-7
