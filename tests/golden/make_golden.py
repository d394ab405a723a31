"""Generate the golden fixtures in this directory from the reference build.

Runs oracle/_ref/cfdv_ref -- the CFDV reference sources compiled unmodified with the
single-rank shims (oracle/Makefile) -- on the small synthetic cases of
cfdv_b200.meshgen.SMALL and stores, per case, what the reference computed:
dt, GMRES tolerance / estimates / final g(m) and the conserved state U after every
step, the RMS line, and the element matrices after ApplyBC for step 0 (all elements
for the 2D lid case, a fixed sample of elements otherwise, to keep files small).

Usage (in a checkout with the reference sources present):
    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from cfdv_b200 import meshgen as mg  # noqa: E402
from oracle import oracle as O  # noqa: E402

STEPS = {"lid8": 3, "plate20": 3, "ramp4": 2, "cyl4": 2, "duct4": 2,
         # the same cases with every third element adaptive (meshgen.adaptive_demo), read by the
         # reference from its "adap" file (control adap = 1)
         "lid8_adap": 3, "plate20_adap": 2, "ramp4_adap": 2, "cyl4_adap": 2}


def make_case(name):
    if name.endswith("_adap"):
        return mg.adaptive_demo(mg.SMALL[name[: -len("_adap")]]())
    return mg.SMALL[name]()


def case_digest(case):
    h = hashlib.sha256()
    h.update(case.nodes.astype("<f8").tobytes())
    h.update(case.elements.astype("<i4").tobytes())
    if case.adap_elements is not None:
        h.update(case.adap_elements.astype("<i4").tobytes())
        h.update(case.adap_hnm.astype("<f8").tobytes())
    return h.hexdigest()


def sample_elements(case, k=12):
    bc = case.bc
    bnd = np.where((bc != 0).any(axis=1))[0]
    inner = np.where((bc == 0).all(axis=1))[0]
    pick = np.concatenate([bnd[:: max(1, len(bnd) // k)][:k], inner[:: max(1, len(inner) // 4)][:4]])
    return np.unique(pick).astype(np.int64)


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    for name, steps in STEPS.items():
        case = make_case(name)
        with tempfile.TemporaryDirectory() as d:
            mg.write_case(case, d)
            rec = O.run_reference(d, os.path.join(d, "out.rec"), steps=steps, dump_step=0)
        out = {"digest": np.array(case_digest(case)), "steps": np.array(steps)}
        for k in ("U_init", "cleng", "dirichlet", "s1234", "dt_dump"):
            out[k] = rec[k]
        Ke = case.nnod * case.neqn
        R = rec["R_bc"].reshape(case.n_elements, Ke, Ke)
        rhs = rec["rhs_bc"].reshape(case.n_elements, Ke)
        el = np.arange(case.n_elements) if name.startswith("lid8") else sample_elements(case)
        if case.adap_elements is not None:  # add adaptive elements to the sample
            el = np.union1d(el, case.adap_elements[: 24]).astype(np.int64)
        out["elements"] = el
        out["R_bc"] = R[el]
        out["rhs_bc"] = rhs[el]
        for s in range(steps):
            for k in ("dt", "tol", "est", "gfinal", "U", "rms"):
                out[f"{k}@{s}"] = rec[f"{k}@{s}"]
        path = os.path.join(here, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(name, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
