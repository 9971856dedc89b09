"""Ragged batches whose large graphs are solved alone by the single-graph
engine (nwgpu_batch_create / nwgpu_pr_ragged, NWGPU_RAGGED_SOLO_ENTRIES).

The bound is lowered here so that small graphs take that path. A graph solved
alone must give exactly what a single-graph handle gives for it (the same
engine on the same CSR: bitwise, the same sweep count); the batch as a whole
must give what the all-in-batch solve gives within the parity tolerance, and
per-graph stats must count the solo graphs' own sweeps.
"""
import numpy as np
import pytest
import torch

from nwgraph_b200 import Graph, GraphBatch, NwgpuError, graphs as G, shard as S
from nwgraph_b200 import _native as N

pytestmark = pytest.mark.gpu

D = 0.85
SOLO = 40000


def batch_graphs():
    gs = []
    for i in range(14):
        if i % 3 == 0:
            gs.append(G.rmat(12, 16, 100 + i))  # about 120K entries: solo
        elif i % 3 == 1:
            gs.append(G.grid(900 + 37 * i))      # small grid: in the batch
        else:
            gs.append(G.rmat(8, 8, 200 + i))     # small RMAT: in the batch
    gs.insert(5, G.CSR(np.zeros(1, np.uint32), np.zeros(0, np.uint32)))  # an empty graph
    return gs


def solve_batch(gs, monkeypatch, solo, launch="graph", device=False, thr=1e-6, iters=200):
    monkeypatch.setenv("NWGPU_RAGGED_SOLO_ENTRIES", str(solo))
    deg = np.concatenate([g.out_degree() for g in gs])
    b0 = GraphBatch.from_graphs([(g.row_ptr, g.col) for g in gs])
    if device:
        dev = torch.device("cuda", 0)
        rp = np.concatenate([g.row_ptr for g in gs])
        cl = np.concatenate([g.col for g in gs])
        b0.release()
        b0 = GraphBatch(b0.vertex_offsets, b0.entry_offsets, torch.from_numpy(rp.view(np.int32)).to(dev),
                        torch.from_numpy(cl.view(np.int32)).to(dev))
        out = torch.empty(len(deg), dtype=torch.float32, device=dev)
        st = b0.page_rank(torch.from_numpy(deg.view(np.int32)).to(dev), out, D, thr, iters, launch=launch)
        out = out.cpu().numpy()
    else:
        out = np.empty(len(deg), np.float32)
        st = b0.page_rank(deg, out, D, thr, iters, launch=launch)
    parts = b0.split(out)
    b0.release()
    return parts, st


def test_solo_graphs_equal_single_graph_handles(gpu, monkeypatch):
    gs = batch_graphs()
    parts, st = solve_batch(gs, monkeypatch, SOLO)
    assert st.converged_graphs == len(gs)
    swept = 0.0
    for i, g in enumerate(gs):
        swept += float(g.nnz) * int(st.graph_iterations[i])
        if g.nnz < SOLO:
            continue
        with Graph(g.row_ptr, g.col) as h:
            r = np.empty(g.n, np.float32)
            s1 = h.page_rank(g.out_degree(), r, D, 1e-6, 200)
        assert np.array_equal(parts[i].view(np.uint32), r.view(np.uint32)), i
        assert int(st.graph_iterations[i]) == s1.iterations and bool(st.graph_converged[i])
        assert st.graph_errors[i] == s1.final_error
    assert st.entries_swept == swept
    assert st.sweeps == int(st.graph_iterations.max())


def test_solo_and_batched_paths_agree(gpu, monkeypatch):
    gs = batch_graphs()
    a, sa = solve_batch(gs, monkeypatch, SOLO)
    b, sb = solve_batch(gs, monkeypatch, 0)  # every graph in the batch
    for i in range(len(gs)):
        d = np.abs(a[i].astype(np.float64) - b[i])
        assert d.max(initial=0.0) <= 1e-6 and d.sum() <= 1e-5, i
        assert abs(int(sa.graph_iterations[i]) - int(sb.graph_iterations[i])) <= 1, i


@pytest.mark.parametrize("launch,device", [("stream", False), ("graph", True)])
def test_launch_modes_and_device_pointers(gpu, monkeypatch, launch, device):
    gs = batch_graphs()
    a, _ = solve_batch(gs, monkeypatch, SOLO)
    b, _ = solve_batch(gs, monkeypatch, SOLO, launch=launch, device=device)
    for i in range(len(gs)):
        assert np.array_equal(a[i].view(np.uint32), b[i].view(np.uint32)), i


def test_graph_shares_equal_the_whole_batch(gpu, monkeypatch):
    monkeypatch.setenv("NWGPU_RAGGED_SOLO_ENTRIES", str(SOLO))
    gs = batch_graphs()
    vo = np.concatenate([[0], np.cumsum([g.n for g in gs])]).astype(np.uint64)
    eo = np.concatenate([[0], np.cumsum([g.nnz for g in gs])]).astype(np.uint64)
    rp = np.concatenate([g.row_ptr for g in gs])
    cl = np.concatenate([g.col for g in gs])
    deg = np.concatenate([g.out_degree() for g in gs])
    whole = np.empty(int(vo[-1]), np.float32)
    with GraphBatch(vo, eo, rp, cl) as bt:
        bt.page_rank(deg, whole, D, 1e-6, 200)
    b = S.graph_bounds(vo, eo, 3)
    for q in range(3):
        lo, hi = int(b[q]), int(b[q + 1])
        if hi == lo:
            continue
        v0, v1 = int(vo[lo]), int(vo[hi])
        part = np.empty(v1 - v0, np.float32)
        with GraphBatch(*S.batch_slice(vo, eo, rp, cl, lo, hi)) as bt:
            bt.page_rank(np.ascontiguousarray(deg[v0:v1]), part, D, 1e-6, 200)
        assert np.array_equal(part.view(np.uint32), whole[v0:v1].view(np.uint32)), q


def test_invalid_solo_graph_rejected(gpu, monkeypatch):
    monkeypatch.setenv("NWGPU_RAGGED_SOLO_ENTRIES", "100")
    ok = G.rmat(6, 4, 1)
    bad = G.rmat(8, 8, 2)
    col = bad.col.copy()
    col[7] = bad.n + 5  # a column id past the graph
    with pytest.raises(NwgpuError) as ei:
        GraphBatch.from_graphs([(ok.row_ptr, ok.col), (bad.row_ptr, col)])
    assert ei.value.status == N.ERR_INVALID_GRAPH and "graph 1" in str(ei.value)


def test_solo_solve_longer_than_one_graph_launch(gpu, monkeypatch):
    """5000 fixed sweeps: the solo graphs' queued loop stops after one CUDA-graph
    launch (4096 sweeps) and finishes on the full loop, with the same bits as a
    single-graph handle."""
    gs = [G.rmat(12, 16, 100), G.grid(900), G.rmat(12, 16, 103)]
    parts, st = solve_batch(gs, monkeypatch, SOLO, thr=0.0, iters=5000)
    assert st.sweeps == 5000
    for i in (0, 2):
        g = gs[i]
        with Graph(g.row_ptr, g.col) as h:
            r = np.empty(g.n, np.float32)
            s1 = h.page_rank(g.out_degree(), r, D, 0.0, 5000)
        assert s1.iterations == 5000 and int(st.graph_iterations[i]) == 5000
        assert np.array_equal(parts[i].view(np.uint32), r.view(np.uint32)), i


@pytest.mark.parametrize("graphs", [[100, 103], [101]])
def test_every_graph_solved_alone(gpu, monkeypatch, graphs):
    """A batch whose graphs are all solved alone: the batch itself has no tiles
    and no entries."""
    gs = [G.rmat(12, 16, s) for s in graphs]
    parts, st = solve_batch(gs, monkeypatch, SOLO)
    assert st.converged_graphs == len(gs)
    for i, g in enumerate(gs):
        with Graph(g.row_ptr, g.col) as h:
            r = np.empty(g.n, np.float32)
            s1 = h.page_rank(g.out_degree(), r, D, 1e-6, 200)
        assert np.array_equal(parts[i].view(np.uint32), r.view(np.uint32)) and int(st.graph_iterations[i]) == s1.iterations
