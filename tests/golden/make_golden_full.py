"""Golden fixtures of the reference build on the full-size synthetic configurations.

Runs oracle/_ref/cfdv_ref (the CFDV reference sources compiled unmodified with the
single-rank shims, oracle/Makefile) on the meshes of cfdv_b200.meshgen.FULL and keeps a
sample of what it computed, small enough to commit:

  plate   2D flat plate 200x100 quad4, M 3, Re 1e4: the reference's own GMRES(30) with one
          restart (its MPI_GMRES) for STEPS["plate"] steps.  Per step: dt, the tolerance,
          every Givens estimate and g(m), the RMS line, U at a fixed sample of unknowns and
          per-field sums of U and U^2 over all nodes; the whole U after the last step;
          R and rhs after ApplyBC at step 0 for a sample of elements.
  ramp    3D compression ramp 128x64x32 hex8 (262,144 elements): the same for
          STEPS["ramp"] steps of the reference's GMRES(50), without the whole-U record.
  cylinder, duct
          3D O-grid cylinder 96x128x16 and the jittered 200x100x50 duct (10^6 elements):
          step 0 only -- CFL over the whole mesh, then FDVGalerkin and ApplyBC on the sampled
          elements alone (cfdv_ref --form-subset); s1..s4 of those elements.

The element sample takes, for every distinct pattern of face boundary codes, the first
and the last element with it, plus evenly spaced interior elements.  The unknown sample is
drawn with numpy's default_rng(20261203).

Usage (in a checkout with the reference sources present, after `make -C oracle ref`):
    python tests/golden/make_golden_full.py [plate] [ramp] [cylinder] [duct]
The reference takes about 0.7 s per plate step, 3 min per ramp step and, for the duct,
about 40 GB of host memory (three Ke x Ke matrices per element).
"""
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)
from cfdv_b200 import meshgen as mg  # noqa: E402
from oracle import oracle as O  # noqa: E402
from make_golden import case_digest  # noqa: E402

STEPS = {"plate": 25, "ramp": 2, "cylinder": 0, "duct": 0}
# unknowns sampled per step (the plate also keeps its whole U after the last step)
DOF_SAMPLE = {"plate": 1024, "ramp": 8192, "cylinder": 8192, "duct": 8192}


def sample_elements_full(case, n_inner=16):
    """First and last element of every distinct face-code pattern, plus interior elements."""
    bc = case.bc
    pats, first = np.unique(bc, axis=0, return_index=True)
    _, last_rev = np.unique(bc[::-1], axis=0, return_index=True)
    last = len(bc) - 1 - last_rev
    inner = np.where((bc == 0).all(axis=1))[0]
    pick = np.concatenate([first, last, inner[:: max(1, len(inner) // n_inner)][:n_inner]])
    return np.unique(pick).astype(np.int32)


def field_sums(U, neqn):
    u = U.reshape(-1, neqn)
    return np.concatenate([u.sum(axis=0), (u * u).sum(axis=0)])


def make(name):
    case = mg.FULL[name]()
    steps = STEPS[name]
    el = sample_elements_full(case)
    rng = np.random.default_rng(mg.SEED)
    n_dof = case.n_nodes * case.neqn
    dofs = np.sort(rng.choice(n_dof, size=min(DOF_SAMPLE[name], n_dof), replace=False)).astype(np.int64)
    t0 = time.time()
    with tempfile.TemporaryDirectory() as d:
        mg.write_case(case, d)
        el_file = os.path.join(d, "elements.i32")
        el.astype("<i4").tofile(el_file)
        extra = ["--elements", el_file] + (["--form-subset"] if steps == 0 else [])
        rec = O.run_reference(d, os.path.join(d, "out.rec"), steps=max(steps, 1), dump_step=0,
                              extra=extra, timeout=4 * 3600)
    wall = time.time() - t0
    Ke = case.nnod * case.neqn
    out = {"digest": np.array(case_digest(case)), "steps": np.array(steps), "elements": el.astype(np.int64),
           "dof_sample": dofs, "dt_dump": rec["dt_dump"], "U_init_sum": field_sums(rec["U_init"], case.neqn),
           "s1234": rec["s1234"].reshape(-1, 4),
           "R_bc": rec["R_bc"].reshape(len(el), Ke, Ke), "rhs_bc": rec["rhs_bc"].reshape(len(el), Ke),
           "wall_s": np.array(wall)}
    if steps == 0:
        out["form_time_s"] = rec["form_time"]
    for s in range(steps):
        U = rec[f"U@{s}"]
        for k in ("dt", "tol", "est", "gfinal", "rms", "steptime"):
            out[f"{k}@{s}"] = rec[f"{k}@{s}"]
        out[f"Usample@{s}"] = U[dofs]
        out[f"Usum@{s}"] = field_sums(U, case.neqn)
    if name == "plate":
        out[f"U@{steps - 1}"] = rec[f"U@{steps - 1}"]
    path = os.path.join(HERE, f"{case.name}.npz")
    np.savez_compressed(path, **out)
    print(name, case.name, os.path.getsize(path), "bytes", f"{wall:.0f} s", flush=True)


def main():
    names = sys.argv[1:] or ["plate", "ramp", "cylinder", "duct"]
    for n in names:
        make(n)


if __name__ == "__main__":
    main()
