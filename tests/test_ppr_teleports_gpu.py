"""Batched personalised PageRank with teleport vectors on an unweighted graph
(nwgpu_ppr_batched_teleports), the teleport-matrix form of the batched call.
No counterpart in the reference:

* one-hot teleports give nwgpu_ppr_batched's columns for those seeds bit for
  bit, with the same sweep counts (the base term (1 - d) * 1 is exact), also in
  batches wide enough to narrow;
* dense teleports (nonnegative, each column summing to 1) on a directed graph
  with dangling vertices give the FP64 fixed point of
  r = (1 - d) t + d A^T D^{-1} r (oracle.pr_f64, leak semantics) to 1e-6;
* a 100-column batch, which narrows, equals 32-column batches bit for bit;
* device pointers and both launch modes give the same bits.
"""
import numpy as np
import pytest

import oracle as O
from nwgraph_b200 import Graph, NwgpuError, graphs as G
from nwgraph_b200 import _native as N

pytestmark = pytest.mark.gpu

D = 0.85


def directed(n=12000, m=150000, seed=8):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, n, m)
    dst = (rng.pareto(1.3, m) * 25).astype(np.int64) % n
    keep = (src < n - 40) & (src != dst)  # the last 40 vertices have no out-edges
    return G.from_edges(dst[keep], src[keep], n)  # rows = in-neighbours


def dense_teleports(n, k, seed):
    rng = np.random.default_rng(seed)
    t = rng.uniform(0.0, 1.0, (n, k))
    t[:, 0] = 1.0  # a uniform column
    return (t / t.sum(axis=0, keepdims=True)).astype(np.float32)


@pytest.mark.parametrize("k", [20, 40, 100])
def test_one_hot_teleports_equal_seed_form(gpu, k):
    g = G.rmat(14, 16, 6)
    deg = g.out_degree()
    seeds = G.random_sources(deg, k, seed=11)
    t = np.zeros((g.n, k), np.float32)
    t[seeds, np.arange(k)] = 1.0
    with Graph(g.row_ptr, g.col) as h:
        a = np.empty((g.n, k), np.float32)
        sa = h.ppr_batched(deg, seeds, a, D, 1e-6, 100)
        b = np.empty((g.n, k), np.float32)
        sb = h.ppr_batched_teleports(deg, t, b, D, 1e-6, 100)
    assert sa.all_converged and sb.all_converged
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(sa.col_iterations, sb.col_iterations) and sa.iterations == sb.iterations


def test_dense_teleports_match_fp64(gpu):
    g = directed()
    deg = g.out_degree()
    t = dense_teleports(g.n, 12, seed=3)
    with Graph(g.row_ptr, g.col) as h:
        out = np.empty(t.shape, np.float32)
        st = h.ppr_batched_teleports(deg, t, out, D, 1e-9, 500)
    assert st.all_converged and len(set(st.col_iterations.tolist())) > 1
    for c in range(t.shape[1]):
        ref, _, _ = O.pr_f64(g.row_ptr, g.col, teleport=t[:, c].astype(np.float64), damping=D, tol=1e-15)
        d = np.abs(out[:, c].astype(np.float64) - ref)
        assert d.max() <= 1e-6 and d.sum() <= 1e-5, (c, d.max(), d.sum())


def test_wide_batch_equals_32_column_batches(gpu):
    g = G.rmat(13, 16, 9)
    deg = g.out_degree()
    t = dense_teleports(g.n, 100, seed=4)
    with Graph(g.row_ptr, g.col) as h:
        whole = np.empty(t.shape, np.float32)
        st = h.ppr_batched_teleports(deg, t, whole, D, 1e-7, 300)
        for c0 in range(0, 100, 32):
            tc = np.ascontiguousarray(t[:, c0:c0 + 32])
            part = np.empty(tc.shape, np.float32)
            sp = h.ppr_batched_teleports(deg, tc, part, D, 1e-7, 300)
            assert np.array_equal(part.view(np.uint32), whole[:, c0:c0 + 32].view(np.uint32)), c0
            assert np.array_equal(sp.col_iterations, st.col_iterations[c0:c0 + 32])


def test_device_pointers_and_launch_modes(gpu):
    import torch
    g = directed(4000, 40000, 2)
    deg = g.out_degree()
    t = dense_teleports(g.n, 40, seed=5)
    with Graph(g.row_ptr, g.col) as h:
        a = np.empty(t.shape, np.float32)
        h.ppr_batched_teleports(deg, t, a, D, 1e-7, 300)
        b = np.empty(t.shape, np.float32)
        h.ppr_batched_teleports(deg, t, b, D, 1e-7, 300, launch="stream")
        od = torch.empty(t.shape, dtype=torch.float32, device="cuda")
        h.ppr_batched_teleports(torch.from_numpy(deg.view(np.int32)).cuda(), torch.from_numpy(t).cuda(), od, D, 1e-7,
                                300)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(a.view(np.uint32), od.cpu().numpy().view(np.uint32))


def test_bad_arguments(gpu):
    g = G.rmat(8, 8, 1)
    deg = g.out_degree()
    with Graph(g.row_ptr, g.col) as h:
        t = np.full((g.n, 129), 1.0 / g.n, np.float32)
        with pytest.raises(NwgpuError) as ei:
            h.ppr_batched_teleports(deg, t, np.empty(t.shape, np.float32))
        assert ei.value.status == N.ERR_INVALID_ARG
        t = np.full((g.n, 2), 1.0 / g.n, np.float32)
        with pytest.raises(NwgpuError) as ei:
            h.ppr_batched_teleports(deg, t, np.empty(t.shape, np.float32), damping_factor=1.5)
        assert ei.value.status == N.ERR_INVALID_ARG
