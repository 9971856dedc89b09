"""Graph construction on the device (nwgpu_csr_from_edges and the edge
generators) against the reference's own build steps.

Golden vectors: csr_build.npz holds the CSRs the reference's
remove_self_loops / lexical sort + uniq / fill_directed / fill_undirected
(build.hpp:58-69, 209-272, 394-410; rows sorted) built from edge lists with
repeated edges, reversed pairs and self-loops, for every flag combination;
the device build must equal them bit for bit (row pointers, columns,
degrees). Larger inputs are checked against the restatement oracle.build_csr
(pinned to those vectors in test_oracle.py), and the device generators
against the host builder they restate.
"""
import numpy as np
import pytest

import oracle as O
from nwgraph_b200 import NwgpuError, construct as K, graphs as G
from nwgraph_b200 import _native as N

pytestmark = pytest.mark.gpu


def test_matches_reference_golden_host_and_device(gpu, csr_golden):
    import torch
    for name, g in csr_golden.items():
        for f in range(0, 0x20, 2):
            csr, deg = K.csr_from_edges(g["src"], g["dst"], g["n"], f)
            ref = g[f]
            assert np.array_equal(csr.row_ptr, ref["row_ptr"]), (name, f)
            assert np.array_equal(csr.col, ref["col"]), (name, f)
            assert np.array_equal(deg, ref["deg"]), (name, f)
            s = torch.from_numpy(g["src"].astype(np.int32)).cuda()
            d = torch.from_numpy(g["dst"].astype(np.int32)).cuda()
            rp, cl, dg = K.csr_from_edges(s, d, g["n"], f)
            assert np.array_equal(rp.cpu().numpy().view(np.uint32), ref["row_ptr"]), (name, f)
            assert np.array_equal(cl.cpu().numpy().view(np.uint32), ref["col"]), (name, f)
            assert np.array_equal(dg.cpu().numpy().view(np.uint32), ref["deg"]), (name, f)


@pytest.mark.parametrize("n,m", [(1, 5), (97, 2000), (100_000, 1_500_000), ((1 << 20) + 3, 3_000_000)])
def test_matches_oracle_all_flags(gpu, n, m):
    rng = np.random.default_rng(n)
    s = rng.integers(0, n, m).astype(np.uint32)
    d = rng.integers(0, n, m).astype(np.uint32)
    s[: m // 20] = d[: m // 20]  # self-loops
    for f in range(0, 0x40, 2):
        csr, deg = K.csr_from_edges(s, d, n, f)
        rp, cl, dg = O.build_csr(s, d, n, f)
        assert np.array_equal(csr.row_ptr, rp) and np.array_equal(csr.col, cl) and np.array_equal(deg, dg), (n, f)


@pytest.mark.parametrize("scale,ef,seed", [(6, 16, 1), (12, 8, 42), (16, 16, 7), (18, 12.5, 3)])
def test_device_rmat_equals_host_builder(gpu, scale, ef, seed):
    host = G.rmat(scale, ef, seed)
    dev = K.rmat(scale, ef, seed)
    assert np.array_equal(dev.row_ptr, host.row_ptr) and np.array_equal(dev.col, host.col)


@pytest.mark.parametrize("n", [1, 2, 5, 1000, 123_456])
def test_device_grid_equals_host_builder(gpu, n):
    host = G.grid(n)
    dev = K.grid(n)
    assert np.array_equal(dev.row_ptr, host.row_ptr) and np.array_equal(dev.col, host.col)


def test_rmat_ids_fold_modulo_n(gpu):
    full_s, full_d = K.rmat_edges(12, 50_000, seed=9)
    s, d = K.rmat_edges(12, 50_000, seed=9, n=3000)
    fs = full_s.cpu().numpy().view(np.uint32)
    fd = full_d.cpu().numpy().view(np.uint32)
    assert np.array_equal(s.cpu().numpy().view(np.uint32), fs % 3000)
    assert np.array_equal(d.cpu().numpy().view(np.uint32), fd % 3000)


def test_errors(gpu):
    s = np.array([0, 1, 7], np.uint32)
    d = np.array([1, 2, 3], np.uint32)
    with pytest.raises(NwgpuError) as ei:
        K.csr_from_edges(s, d, 5)  # endpoint 7 >= n
    assert ei.value.status == N.ERR_INVALID_GRAPH
    import ctypes as C
    rp = np.empty(9, np.uint32)
    cl = np.empty(2, np.uint32)
    nnz = C.c_uint64()
    st = N.lib().nwgpu_csr_from_edges(s.ctypes.data, d.ctypes.data, 3, 8, K.UNDIRECTED, rp.ctypes.data, cl.ctypes.data,
                                      2, C.byref(nnz), None, None)
    assert st == N.ERR_INVALID_ARG and nnz.value == 6  # capacity 2 < 6 entries: refused, size reported
    with pytest.raises(NwgpuError):
        K.rmat_edges(0, 10)


def test_load_graph_from_files(gpu):
    """load_graph: a graph file's edges built into adjacency<1> on the device,
    as the reference driver's load_graph + build_adjacency<1> (rows sorted)."""
    import os
    files = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "files")
    for name in ("general_real.mtx", "symmetric_pattern.mtx", "karate_pattern.mtx", "general_ref.nw"):
        csr, deg = K.load_graph(os.path.join(files, name))
        s, d, n = K.read_edges(os.path.join(files, name))
        rp, cl, dg = O.build_csr(s, d, n, 0)
        assert np.array_equal(csr.row_ptr, rp) and np.array_equal(csr.col, cl) and np.array_equal(deg, dg), name
