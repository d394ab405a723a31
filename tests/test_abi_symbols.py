"""The C-ABI library loads without a GPU and exports every declared entry point."""
import ctypes
import os
import re

from conftest import ROOT

from cfdv_b200 import gpu


def declared_functions():
    src = open(os.path.join(ROOT, "include", "cfdv_gpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(cfdv_\w+)\s*\(", src, re.M)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(gpu.EXPORTS)


def test_library_exports_every_symbol():
    lib = ctypes.CDLL(gpu.LIB_PATH)
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_no_gpu_fails_loudly_or_runs(monkeypatch):
    # without a CUDA device the constructor must raise, never fall back to the CPU
    import torch
    if torch.cuda.is_available():
        return
    from conftest import get_case
    try:
        gpu.FDVSolver(get_case("lid8"))
    except gpu.CfdvError as e:
        assert e.code in (2,)
    else:
        raise AssertionError("FDVSolver ran without a GPU")
