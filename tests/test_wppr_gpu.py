"""Weighted personalised PageRank for many teleport vectors at once
(nwgpu_wppr_batched): the batched variant of the weighted configuration (16
teleport vectors). No counterpart in the reference: every column must give
what nwgpu_wpr_run gives for that teleport vector alone (1e-6 max-abs, its
own stopping sweep within one) and the FP64 oracle's fixed point (1e-6)."""
import numpy as np
import pytest

import oracle as O
from nwgraph_b200 import Graph, NwgpuError, graphs as G
from nwgraph_b200 import _native as N

pytestmark = pytest.mark.gpu

D = 0.85


@pytest.fixture(scope="module")
def case():
    g = G.rmat(13, 16, 21)
    w = G.edge_weights(g.nnz, seed=1234)
    rng = np.random.default_rng(99)
    k = 16
    t = rng.uniform(0.0, 1.0, (g.n, k))
    t[:, 0] = 1.0  # column 0: uniform teleport
    t[:, 1] = 0.0  # column 1: one-hot
    t[17, 1] = 1.0
    t = (t / t.sum(axis=0, keepdims=True)).astype(np.float32)
    return g, w, t


def test_columns_match_single_solves_and_fp64(gpu, case):
    g, w, t = case
    k = t.shape[1]
    with Graph(g.row_ptr, g.col, weights=w) as h:
        out = np.empty((g.n, k), np.float32)
        st = h.weighted_page_rank_batched(t, out, D, 1e-7, 500)
        assert st.all_converged and st.col_converged.all()
        assert len(set(st.col_iterations.tolist())) > 1  # columns stop at their own sweeps
        for c in range(k):
            r1 = np.empty(g.n, np.float32)
            s1 = h.weighted_page_rank(np.ascontiguousarray(t[:, c]), r1, D, 1e-7, 500)
            assert abs(int(st.col_iterations[c]) - s1.iterations) <= 1, c
            assert np.abs(out[:, c] - r1).max() <= 1e-6, c
            ref, _, _ = O.pr_f64(g.row_ptr, g.col, weights=w, teleport=t[:, c].astype(np.float64), damping=D,
                                 tol=1e-15)
            assert np.abs(out[:, c] - ref).max() <= 1e-6, c


def test_device_pointers_and_launch_modes(gpu, case):
    import torch
    g, w, t = case
    with Graph(g.row_ptr, g.col, weights=w) as h:
        a = np.empty(t.shape, np.float32)
        h.weighted_page_rank_batched(t, a, D, 1e-6, 300)
        b = np.empty(t.shape, np.float32)
        h.weighted_page_rank_batched(t, b, D, 1e-6, 300, launch="stream")
        td = torch.from_numpy(t).cuda()
        od = torch.empty(t.shape, dtype=torch.float32, device="cuda")
        h.weighted_page_rank_batched(td, od, D, 1e-6, 300)
        # the unweighted batched solve on the same handle still runs (its own kernels)
        deg = g.out_degree()
        seeds = np.array([1, 5, 9], np.uint32)
        pp = np.empty((g.n, 3), np.float32)
        h.ppr_batched(deg, seeds, pp, D, 1e-6, 100)
        ref, _, _ = O.ppr_jacobi_f32(g.row_ptr, g.col, deg, 5, D, 1e-6, 100)
        assert np.abs(pp[:, 1] - ref).max() <= 1e-6
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(a.view(np.uint32), od.cpu().numpy().view(np.uint32))


def test_unweighted_graph_rejected(gpu, case):
    g, w, t = case
    with Graph(g.row_ptr, g.col) as h:
        with pytest.raises(NwgpuError) as ei:
            h.weighted_page_rank_batched(t, np.empty(t.shape, np.float32))
        assert ei.value.status == N.ERR_UNSUPPORTED
