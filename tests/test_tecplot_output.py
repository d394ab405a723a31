"""The host Tecplot writer (cfdv_b200/host/cfdv_host.hpp) against the reference's own
MPI_TecplotOut (Utility/IO/MPI_TecplotOut.h), byte for byte, on the initial state."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, get_case

REF = os.path.join(ROOT, "oracle", "_ref", "cfdv_ref")
EMIT = os.path.join(ROOT, "tests", "emu", "tecplot_emit")


@pytest.fixture(scope="module")
def emit():
    src = os.path.join(ROOT, "tests", "emu", "tecplot_emit.cpp")
    hdr = os.path.join(ROOT, "cfdv_b200", "host", "cfdv_host.hpp")
    if not os.path.exists(EMIT) or os.path.getmtime(EMIT) < max(os.path.getmtime(src), os.path.getmtime(hdr)):
        subprocess.run(["g++", "-std=c++17", "-O2", src, "-o", EMIT], check=True)
    return EMIT


@pytest.mark.skipif(not os.path.exists(REF), reason="reference build oracle/_ref not present")
@pytest.mark.parametrize("name", ["lid8", "plate20", "ramp4"])
def test_tecplot_matches_reference_writer(emit, oracle_lib, name):
    from cfdv_b200 import meshgen as mg
    case = get_case(name)
    o = oracle_lib.Oracle(case)
    U = o.init_U()
    s = o.fdvparam(U)
    with tempfile.TemporaryDirectory() as d:
        cdir = os.path.join(d, "case")
        mg.write_case(case, cdir)
        rdir, mdir = os.path.join(d, "ref"), os.path.join(d, "mine")
        os.makedirs(rdir)
        os.makedirs(mdir)
        subprocess.run([REF, cdir, os.path.join(d, "r.rec"), "--steps", "1", "--tecplot", "--quiet"], cwd=rdir,
                       check=True, stdin=subprocess.DEVNULL)
        U.tofile(os.path.join(d, "U.bin"))
        s.tofile(os.path.join(d, "s.bin"))
        subprocess.run([emit, cdir, os.path.join(d, "U.bin"), os.path.join(d, "s.bin"), "0", "0", mdir], check=True)
        ref = open(os.path.join(rdir, "tecplot_0.plt"), "rb").read()
        mine = open(os.path.join(mdir, "tecplot_0.plt"), "rb").read()
    assert mine == ref


def test_tecplot_file_name():
    # to_string<double>(iter) as in MPI_TecplotOut.h:189
    src = '#include "../../cfdv_b200/host/cfdv_host.hpp"\n#include <cstdio>\nint main(){for(int i: {0,100,123400,1000000}) printf("%s\\n", cfdv_host::tecplot_name(i).c_str());}'
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(ROOT, "tests", "emu", "_name_probe.cpp")
        open(p, "w").write(src)
        try:
            subprocess.run(["g++", "-std=c++17", p, "-o", os.path.join(d, "a")], check=True)
            out = subprocess.run([os.path.join(d, "a")], capture_output=True, text=True, check=True).stdout.split()
        finally:
            os.remove(p)
    assert out == ["tecplot_0.plt", "tecplot_100.plt", "tecplot_123400.plt", "tecplot_1e+06.plt"]
