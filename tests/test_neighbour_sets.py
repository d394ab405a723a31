"""The neighbour sets of the persistent GMRES solve (cfdv_b200/csrc/neighbour_sets.h), built on
the CPU by tests/emu/nbr_emu.cpp, against the data dependences they stand for.  In the 2D
delayed-CGS2 step, block b's element pass reads x at the nodes of its elements and its node
pass reads the products of the elements at its nodes; before each, b waits only for the
blocks that write those.  A set that missed a writer would let b read stale data, so each set
must equal the writers exactly (b itself excluded)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, get_case

EMU = os.path.join(ROOT, "tests", "emu", "libnbr_emu.so")


@pytest.fixture(scope="module")
def emu():
    src = os.path.join(ROOT, "tests", "emu", "nbr_emu.cpp")
    hdr = os.path.join(ROOT, "cfdv_b200", "csrc", "neighbour_sets.h")
    if not os.path.exists(EMU) or os.path.getmtime(EMU) < max(os.path.getmtime(src), os.path.getmtime(hdr)):
        subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", src, "-o", EMU], check=True)
    L = C.CDLL(EMU)
    P, I = C.c_void_p, C.c_int
    L.emu_neighbour_sets.argtypes = [I, I, I, P, P, P, I, P, P, I]
    L.emu_neighbour_sets.restype = I
    return L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def node_csr(conn, n_nodes):
    """node -> (element, local node) entries in element order."""
    nnod = conn.shape[1]
    ptr = np.zeros(n_nodes + 1, np.int32)
    np.add.at(ptr, conn.ravel() + 1, 1)
    ptr = np.cumsum(ptr).astype(np.int32)
    idx = np.zeros(conn.size, np.int32)
    fill = ptr[:-1].copy()
    for e in range(conn.shape[0]):
        for l in range(nnod):
            n = conn[e, l]
            idx[fill[n]] = e * nnod + l
            fill[n] += 1
    return ptr, idx


def build(L, case, blocks):
    conn = np.ascontiguousarray(case.conn, dtype=np.int32)
    ptr, idx = node_csr(conn, case.n_nodes)
    out_ptr = np.zeros(2 * (blocks + 1), np.int32)
    out_idx = np.zeros(64 * blocks, np.int32)
    n = L.emu_neighbour_sets(case.ndim, case.n_nodes, case.n_elements, _p(conn), _p(ptr), _p(idx), blocks,
                             _p(out_ptr), _p(out_idx), out_idx.size)
    return n, out_ptr, out_idx[: max(n, 0)], conn


def expected(case, conn, blocks):
    """The writers each block's two gathers depend on, from the solve's ownership."""
    pn = -(-case.n_nodes // blocks)
    per = -(-case.n_elements // blocks)
    xs = [set() for _ in range(blocks)]  # owners of the nodes of b's elements
    ys = [set() for _ in range(blocks)]  # owners of the elements at b's nodes
    for e in range(case.n_elements):
        eb = e // per
        for n in conn[e]:
            nb_ = n // pn
            xs[eb].add(nb_)
            ys[nb_].add(eb)
    return ([s - {b} for b, s in enumerate(xs)], [s - {b} for b, s in enumerate(ys)])


@pytest.mark.parametrize("name", ["lid8", "lid32", "plate20", "lid8_adap"])
@pytest.mark.parametrize("blocks", [148, 37, 5])
def test_sets_equal_the_writers(emu, name, blocks):
    case = get_case(name)
    n, ptr, idx, conn = build(emu, case, blocks)
    assert n >= 0
    xs, ys = expected(case, conn, blocks)
    for b in range(blocks):
        got_x = idx[ptr[b]:ptr[b + 1]]
        got_y = idx[ptr[blocks + 1 + b]:ptr[blocks + 2 + b]]
        assert len(set(got_x)) == len(got_x) and len(set(got_y)) == len(got_y)  # no repeats
        assert set(got_x.tolist()) == xs[b]
        assert set(got_y.tolist()) == ys[b]


def test_flat_plate_sets_are_small(emu):
    from cfdv_b200 import meshgen as mg
    case = mg.plate(200, 100)
    n, ptr, idx, conn = build(emu, case, 148)
    assert n >= 0
    sizes = np.diff(ptr[: 149]).tolist() + np.diff(ptr[149:]).tolist()
    assert max(sizes) <= 3  # the plate's blocks read from at most three others


def test_3d_keeps_grid_barriers(emu):
    n, _, _, _ = build(emu, get_case("ramp4"), 148)
    assert n == -1


def test_scattered_numbering_keeps_grid_barriers(emu):
    """With nodes numbered at random, a block's elements touch nodes of most blocks: the sets
    exceed 32 blocks and the solve falls back to grid barriers."""
    from cfdv_b200 import meshgen as mg
    case = mg.plate(200, 100)
    rng = np.random.default_rng(3)
    perm = rng.permutation(case.n_nodes).astype(np.int32)

    class Scattered:
        ndim, n_nodes, n_elements = case.ndim, case.n_nodes, case.n_elements
        conn = perm[np.asarray(case.conn)]

    n, _, _, _ = build(emu, Scattered, 148)
    assert n == -1
