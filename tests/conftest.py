import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from cfdv_b200 import meshgen as mg  # noqa: E402

SMALL_CASES = ["lid8", "plate20", "ramp4", "cyl4", "duct4"]
ADAPTIVE_CASES = ["lid8_adap", "plate20_adap", "ramp4_adap", "cyl4_adap"]  # every third element with an Hnm
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libcfdv_gpu.so")


_cases = {}


def get_case(name):
    """A small synthetic case; "<name>_adap" is the case with every third element adaptive
    (meshgen.adaptive_demo: hanging-node Hnm matrices)."""
    if name not in _cases:
        if name.endswith("_adap"):
            _cases[name] = mg.adaptive_demo(get_case(name[: -len("_adap")]))
        else:
            _cases[name] = mg.SMALL[name]()
    return _cases[name]


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def rel_err(a, b):
    """max |a - b| / max |b| (0 when both vanish)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.abs(b).max() if b.size else 0.0
    d = np.abs(a - b).max() if b.size else 0.0
    return d / s if s > 0 else d


def elem_rel_err(R, Rref):
    """max over elements of |R_e - Rref_e|_max / |Rref_e|_max."""
    axes = tuple(range(1, Rref.ndim))
    scale = np.abs(Rref).max(axis=axes)
    scale[scale == 0] = 1.0
    return float((np.abs(R - Rref).max(axis=axes) / scale).max())


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O
    if not os.path.exists(O.LIB_PATH):
        O.build()
    return O
