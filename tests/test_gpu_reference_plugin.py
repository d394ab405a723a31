"""The B200 plug-ins inside the reference's own step loop.

oracle/_ref/cfdv_ref_gpu is the reference's driver loop (load, CalcLength, ClearElement,
NodeUnpack, CFL, RMS: the CFDV sources compiled unmodified) with the plug-ins of
cfdv_b200/host/cfdv_reference_plugin.hpp compiled in: `--gpu-solver` puts CudaGMRES, a
GMRESbase, where the reference creates MPI_GMRES (GMRESbase.h:8-23,
MPIBinaryConfiguration.h:123); `--gpu-form` adds GpuFormation in place of the FDVGalerkin
and ApplyBC passes (main.cpp:185-194).  Both runs must reproduce the all-CPU reference
(oracle/_ref/cfdv_ref) on the same case: dt, every Givens estimate the solver prints, g(m)
and U after every step, to <= 1e-10 relative -- the parity bar of the FP64 path."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, get_case, rel_err

from cfdv_b200 import meshgen as mg

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref", "cfdv_ref")
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "cfdv_ref_gpu")
STEPS = 3


def run(binary, case_dir, out, *flags):
    from oracle import oracle as O
    subprocess.run([binary, case_dir, out, "--steps", str(STEPS), "--quiet", *flags], check=True,
                   stdin=subprocess.DEVNULL, timeout=600)
    return O.read_records(out)


@pytest.mark.skipif(not (os.path.exists(REF) and os.path.exists(REF_GPU)),
                    reason="reference build (oracle/_ref) not present: it is made where the reference sources are")
@pytest.mark.parametrize("name", ["lid8", "plate20", "ramp4", "lid8_adap"])
@pytest.mark.parametrize("flags", [("--gpu-solver",), ("--gpu-solver", "--gpu-form")], ids=["solver", "solver+form"])
def test_plugins_in_reference_loop_match_cpu_reference(tmp_path, name, flags):
    case = get_case(name)
    d = str(tmp_path / "case")
    mg.write_case(case, d)
    cpu = run(REF, d, str(tmp_path / "cpu.rec"))
    gpu = run(REF_GPU, d, str(tmp_path / "gpu.rec"), *flags)
    for k in range(STEPS):
        assert gpu[f"dt@{k}"][0] == pytest.approx(cpu[f"dt@{k}"][0], rel=1e-12)
        assert gpu[f"tol@{k}"][0] == pytest.approx(cpu[f"tol@{k}"][0], rel=1e-12)
        assert len(gpu[f"est@{k}"]) == len(cpu[f"est@{k}"])
        assert rel_err(gpu[f"est@{k}"], cpu[f"est@{k}"]) <= 1e-10
        scale = np.abs(cpu[f"est@{k}"]).max()
        assert np.abs(gpu[f"gfinal@{k}"] - cpu[f"gfinal@{k}"]).max() <= 1e-10 * scale
        assert rel_err(gpu[f"U@{k}"], cpu[f"U@{k}"]) <= 1e-10
