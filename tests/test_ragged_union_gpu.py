"""Ragged batches solved as union graphs (the default): the graphs kept in the
batch, in batch order, are cut into groups of at most
NWGPU_RAGGED_UNION_VERTICES vertices, each group the diagonal blocks of one
relabelled CSR swept by the degree-binned kernel, each graph stopping at its
own first sweep below the threshold.

A row's sum depends only on its own entries and length, so each graph must
get, bit for bit and with the same sweep count, what a single-graph handle
gives it; the per-graph L1 changes are summed in another order than a single
handle's (FP64, the same to about 1e-16). The merge-path batch sweep
(NWGPU_RAGGED_UNION=0) must agree within the parity tolerance; both launch
modes and graph shares must give the same bits.
"""
import numpy as np
import pytest

import oracle as O
from nwgraph_b200 import Graph, GraphBatch, graphs as G

pytestmark = pytest.mark.gpu

D = 0.85


def graphs():
    gs = []
    for i in range(24):
        if i % 4 == 0:
            gs.append(G.rmat(11 + (i % 3), 8 + (i % 5) * 4, 300 + i))
        elif i % 4 == 1:
            gs.append(G.grid(400 + 97 * i))
        elif i % 4 == 2:
            gs.append(G.rmat(7, 16, 400 + i))
        else:
            gs.append(G.rmat(14, 16, 500 + i))  # hub rows of more than 2048 entries: chunked long rows
    gs.insert(3, G.CSR(np.zeros(1, np.uint32), np.zeros(0, np.uint32)))      # no vertices
    gs.insert(7, G.CSR(np.zeros(6, np.uint32), np.zeros(0, np.uint32)))      # five vertices, no entries
    gs.insert(11, G.CSR(np.zeros(2, np.uint32), np.zeros(0, np.uint32)))     # one vertex
    return gs


@pytest.fixture(scope="module")
def batch_graphs():
    return graphs()


def solve(gs, thr=1e-6, iters=200, launch="graph"):
    deg = np.concatenate([g.out_degree() for g in gs])
    b = GraphBatch.from_graphs([(g.row_ptr, g.col) for g in gs])
    out = np.empty(len(deg), np.float32)
    st = b.page_rank(deg, out, D, thr, iters, launch=launch)
    parts = b.split(out)
    b.release()
    return parts, st


@pytest.mark.parametrize("thr,iters,vmax", [(1e-6, 200, None), (0.0, 15, None), (1e-6, 200, "5000")])
def test_union_graphs_equal_single_graph_handles(gpu, monkeypatch, batch_graphs, thr, iters, vmax):
    """One union of all graphs, or (vmax 5000) unions of at most 5,000 vertices each, on several streams."""
    monkeypatch.setenv("NWGPU_RAGGED_SOLO_ENTRIES", "0")  # every graph in a union
    if vmax:
        monkeypatch.setenv("NWGPU_RAGGED_UNION_VERTICES", vmax)
    parts, st = solve(batch_graphs, thr, iters)
    for i, g in enumerate(batch_graphs):
        if g.n < 2:  # single-graph handles of 0 or 1 vertices keep the input order (no binned plan)
            continue
        with Graph(g.row_ptr, g.col) as h:
            r = np.empty(g.n, np.float32)
            s1 = h.page_rank(g.out_degree(), r, D, thr, iters)
        assert np.array_equal(parts[i].view(np.uint32), r.view(np.uint32)), i
        assert int(st.graph_iterations[i]) == s1.iterations, i
        assert bool(st.graph_converged[i]) == s1.converged, i
        assert abs(st.graph_errors[i] - s1.final_error) <= 1e-12 * max(1.0, s1.final_error), i


def test_union_agrees_with_the_merge_path_batch_and_the_oracle(gpu, monkeypatch, batch_graphs):
    """Both batch engines stop each graph within one sweep of each other (their row sums round differently) and
    stay within parity of page_rank_v10 restated."""
    monkeypatch.setenv("NWGPU_RAGGED_SOLO_ENTRIES", "0")
    pu, su = solve(batch_graphs)
    monkeypatch.setenv("NWGPU_RAGGED_UNION", "0")
    pm, sm = solve(batch_graphs)
    assert su.converged_graphs == sm.converged_graphs == len(batch_graphs)
    for i, g in enumerate(batch_graphs):
        assert abs(int(su.graph_iterations[i]) - int(sm.graph_iterations[i])) <= 1, i
        if g.n == 0:
            continue
        ref, it, _ = O.jacobi_f32(g.row_ptr, g.col, g.out_degree(), D, 0.0, int(su.graph_iterations[i]))
        d = np.abs(pu[i].astype(np.float64) - ref)
        assert d.max() <= 1e-6 and d.sum() <= 1e-5, i
        d = np.abs(pu[i].astype(np.float64) - pm[i])
        assert d.max() <= 2e-6, i


def test_union_launch_modes_and_shares_bitwise(gpu, monkeypatch, batch_graphs):
    monkeypatch.setenv("NWGPU_RAGGED_SOLO_ENTRIES", "0")
    pa, sa = solve(batch_graphs, launch="graph")
    pb, sb = solve(batch_graphs, launch="stream")
    for x, y in zip(pa, pb):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    assert np.array_equal(sa.graph_iterations, sb.graph_iterations)
    # the first half and the second half as batches of their own
    h = len(batch_graphs) // 2
    p1, _ = solve(batch_graphs[:h])
    p2, _ = solve(batch_graphs[h:])
    for x, y in zip(pa, p1 + p2):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_union_with_solo_graphs(gpu, monkeypatch, batch_graphs):
    """Graphs of at least 200,000 entries solved alone beside the union: both engines give each graph a
    single-graph handle's ranks, bit for bit."""
    monkeypatch.setenv("NWGPU_RAGGED_SOLO_ENTRIES", "200000")
    parts, st = solve(batch_graphs)
    assert st.converged_graphs == len(batch_graphs)
    assert any(g.nnz >= 200000 for g in batch_graphs) and any(0 < g.nnz < 200000 for g in batch_graphs)
    for i, g in enumerate(batch_graphs):
        if g.n < 2:
            continue
        with Graph(g.row_ptr, g.col) as h:
            r = np.empty(g.n, np.float32)
            s1 = h.page_rank(g.out_degree(), r, D, 1e-6, 200)
        assert np.array_equal(parts[i].view(np.uint32), r.view(np.uint32)), i
        assert int(st.graph_iterations[i]) == s1.iterations, i
