"""cfdv_ebe_matvec_static, the EBE product that allocates no device memory.

Some callers of this library may not allocate device memory: an application whose own
memory pool already holds the GPU's free memory (a cudaMalloc from the library would
fail), or code that cannot take the device-wide synchronisation of cudaFree between its
other streams' work.  They pass their own device buffers to cfdv_ebe_matvec_static, which
keeps its element products in a static device array inside the library.  These tests
check it against cfdv_matvec (a context's product, same tolerance as the other EBE-product
tests) on consecutive calls, and that it rejects meshes larger than its fixed scratch.

The file name sorts last, so a run that stops at the first failure has already run every
other test when it gets here; the GPU tests also pass when this file runs on its own."""
import ctypes as C

import numpy as np
import pytest

from conftest import get_case, rel_err

from cfdv_b200 import gpu as G
from cfdv_b200 import meshgen as mg

MAX_DOUBLES = 2097152  # CFDV_STATIC_SCRATCH_DOUBLES in include/cfdv_gpu.h
ERR_ARG, ERR_TOO_LARGE = 1, 8


def node_csr(conn, n_nodes):
    """node -> (element, local node) lists: entries e*nnod + l, increasing within a node."""
    flat = np.ascontiguousarray(conn, dtype=np.int64).ravel()
    ptr = np.zeros(n_nodes + 1, dtype=np.int32)
    ptr[1:] = np.cumsum(np.bincount(flat, minlength=n_nodes))
    idx = np.argsort(flat, kind="stable").astype(np.int32)
    return ptr, idx


def load_case(name):
    return get_case(name) if name in mg.SMALL else mg.FULL[name]()


def test_node_csr_lists_every_element_node_once():
    case = get_case("ramp4")
    ptr, idx = node_csr(case.conn, case.n_nodes)
    flat = case.conn.ravel()
    assert ptr[-1] == flat.size and np.all(np.diff(ptr) >= 0)
    for n in range(case.n_nodes):
        ent = idx[ptr[n]:ptr[n + 1]]
        assert np.all(np.diff(ent) > 0) and np.all(flat[ent] == n)


def test_static_matvec_rejects_oversize_and_bad_arguments():
    """Checked on the host before any GPU work, so this runs without a device."""
    L = G.lib()
    dummy_i = np.zeros(64, dtype=np.int32)
    dummy_d = np.zeros(64)
    pi, pd = dummy_i.ctypes.data, dummy_d.ctypes.data
    y = np.zeros(64)
    py = y.ctypes.data
    # 2D: Ke = 16, 3D: Ke = 40
    assert L.cfdv_ebe_matvec_static(2, 100, MAX_DOUBLES // 16 + 1, pi, pi, pi, pd, pd, py, 0, None) == ERR_TOO_LARGE
    assert L.cfdv_ebe_matvec_static(3, 100, MAX_DOUBLES // 40 + 1, pi, pi, pi, pd, pd, py, 0, None) == ERR_TOO_LARGE
    assert L.cfdv_ebe_matvec_static(4, 100, 10, pi, pi, pi, pd, pd, py, 0, None) == ERR_ARG
    assert L.cfdv_ebe_matvec_static(2, 0, 10, pi, pi, pi, pd, pd, py, 0, None) == ERR_ARG
    assert L.cfdv_ebe_matvec_static(2, 100, 10, None, pi, pi, pd, pd, py, 0, None) == ERR_ARG
    assert L.cfdv_ebe_matvec_static(2, 100, 10, pi, pi, pi, pd, py, py, 0, None) == ERR_ARG


def test_static_matvec_source_allocates_nothing():
    import os
    from conftest import ROOT
    src = open(os.path.join(ROOT, "cfdv_b200", "csrc", "noalloc.cu")).read()
    code = "\n".join(line.split("//")[0] for line in src.splitlines())
    for call in ("cudaMalloc", "cudaFree", "cudaMallocAsync", "cudaFreeAsync", "cudaMallocHost", "new ", "malloc("):
        assert call not in code, call


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["lid8", "plate20", "ramp4", "cyl4", "plate"])
def test_static_matvec_matches_context_matvec(name):
    import torch

    case = load_case(name)
    rng = np.random.default_rng(11)
    with G.FDVSolver(case) as s:
        s.load_node_records()
        s.form(s.cfl(float(case.control["cfl"])))
        R, _ = s.element_matrices()  # raw buffer is the column-major-per-element layout
        xs = [rng.standard_normal(s.n_dof) for _ in range(2)]
        calls = [(xs[0], 0), (xs[1], 0), (xs[1], 1)]
        want = [s.matvec(x, transpose=bool(tr)) for x, tr in calls]
    n_dof = case.n_nodes * (case.ndim + 2)

    dev = torch.device("cuda:0")
    side = torch.cuda.Stream(dev)
    ptr, idx = node_csr(case.conn, case.n_nodes)

    def to_dev(a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype).ravel()).to(dev)

    conn_d, ptr_d, idx_d = to_dev(case.conn, np.int32), to_dev(ptr, np.int32), to_dev(idx, np.int32)
    R_d = to_dev(R, np.float64)
    x_d = [to_dev(x, np.float64) for x, _ in calls]
    y_d = torch.full((n_dof,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    L = G.lib()
    got = []
    for (_, tr), xd in zip(calls, x_d):
        with torch.cuda.stream(side):
            y_d.fill_(float("nan"))
            rc = L.cfdv_ebe_matvec_static(case.ndim, case.n_nodes, case.n_elements, conn_d.data_ptr(),
                                          ptr_d.data_ptr(), idx_d.data_ptr(), R_d.data_ptr(), xd.data_ptr(),
                                          y_d.data_ptr(), tr, C.c_void_p(side.cuda_stream))
            assert rc == 0, G.STATUS.get(rc, rc)
        side.synchronize()
        got.append(y_d.cpu().numpy().copy())

    for g, w in zip(got, want):
        assert np.all(np.isfinite(g))
        assert rel_err(g, w) <= 1e-12


@pytest.mark.gpu
def test_static_matvec_rejects_host_memory_and_leaves_y_alone():
    """Host memory (pageable or pinned) in place of a device buffer is CFDV_ERR_ARG, and a
    mesh above the scratch limit is CFDV_ERR_TOO_LARGE: both before any GPU work, so the
    caller's y keeps what it held."""
    import torch

    case = get_case("lid8")
    n_dof = case.n_nodes * 4
    ptr, idx = node_csr(case.conn, case.n_nodes)
    dev = torch.device("cuda:0")

    def to_dev(a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype).ravel()).to(dev)

    conn_d, ptr_d, idx_d = to_dev(case.conn, np.int32), to_dev(ptr, np.int32), to_dev(idx, np.int32)
    R_d = torch.zeros(case.n_elements * 256, dtype=torch.float64, device=dev)
    x_d = torch.ones(n_dof, dtype=torch.float64, device=dev)
    y_d = torch.full((n_dof,), float("nan"), dtype=torch.float64, device=dev)
    x_pageable = np.ones(n_dof)
    x_pinned = torch.ones(n_dof, dtype=torch.float64).pin_memory()
    L = G.lib()

    def call(n_el, x_ptr, R_ptr=None):
        return L.cfdv_ebe_matvec_static(2, case.n_nodes, n_el, conn_d.data_ptr(), ptr_d.data_ptr(), idx_d.data_ptr(),
                                        R_ptr or R_d.data_ptr(), x_ptr, y_d.data_ptr(), 0, None)

    torch.cuda.synchronize()
    assert call(case.n_elements, x_pageable.ctypes.data) == ERR_ARG
    assert call(case.n_elements, x_pinned.data_ptr()) == ERR_ARG
    R_host = np.zeros(case.n_elements * 256)
    assert call(case.n_elements, x_d.data_ptr(), R_host.ctypes.data) == ERR_ARG
    assert call(MAX_DOUBLES // 16 + 1, x_d.data_ptr()) == ERR_TOO_LARGE
    torch.cuda.synchronize()
    assert torch.isnan(y_d).all()
    # a valid call after the rejected ones works (zero matrices: y = 0)
    assert call(case.n_elements, x_d.data_ptr()) == 0
    torch.cuda.synchronize()
    assert torch.count_nonzero(y_d).item() == 0
