"""Batches sharded over ranks with no exchange per sweep (nwgraph_b200.shard),
on one GPU.

* personalised columns: each rank's share of the seeds (even_bounds), solved
  as a batch of its own, equals those columns of the whole batch bit for bit
  (a converged column is frozen and no column's sums depend on another's),
  for 1 to 5 emulated ranks;
* ragged graphs: each rank's graphs (graph_bounds, batch_slice), solved as a
  batch of their own, equal those graphs of the whole batch bit for bit;
* the torch.distributed entry points (ppr_batched, ShardedBatch) over a
  one-rank NCCL group return the whole result.

The emulated ranks solve one after another in this process: no kernel waits
on another.
"""
import numpy as np
import pytest
import torch

from nwgraph_b200 import Graph, GraphBatch, graphs as G, shard as S

pytestmark = pytest.mark.gpu

D = 0.85


@pytest.fixture(scope="module")
def ppr_case():
    g = G.rmat(14, 16, 2)
    deg = g.out_degree()
    return g, deg, G.random_sources(deg, 40, seed=7)


def ragged_arrays():
    graphs = [G.rmat(12, 16, 1), G.grid(20000), G.rmat(10, 8, 2), G.grid(3000), G.rmat(13, 12, 3),
              G.grid(50000), G.rmat(9, 32, 4), G.rmat(11, 16, 5)]
    vo = np.concatenate([[0], np.cumsum([g.n for g in graphs])]).astype(np.uint64)
    eo = np.concatenate([[0], np.cumsum([g.nnz for g in graphs])]).astype(np.uint64)
    deg = np.concatenate([g.out_degree() for g in graphs])
    return vo, eo, np.concatenate([g.row_ptr for g in graphs]), np.concatenate([g.col for g in graphs]), deg


def whole_ppr(g, deg, seeds):
    out = np.empty((g.n, len(seeds)), np.float32)
    with Graph(g.row_ptr, g.col) as h:
        st = h.ppr_batched(deg, seeds, out, D, 1e-6, 100)
    return out, st


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_column_shares_equal_the_whole_batch(gpu, ppr_case, world):
    g, deg, seeds = ppr_case
    whole, st = whole_ppr(g, deg, seeds)
    assert st.all_converged
    b = S.even_bounds(len(seeds), world)
    with Graph(g.row_ptr, g.col) as h:
        for q in range(world):
            lo, hi = int(b[q]), int(b[q + 1])
            part = np.empty((g.n, hi - lo), np.float32)
            sq = S.solve_columns(h, deg, seeds, part, b, q, D, 1e-6, 100)
            assert np.array_equal(part.view(np.uint32), whole[:, lo:hi].view(np.uint32)), (world, q)
            assert np.array_equal(sq.col_iterations, st.col_iterations[lo:hi])


@pytest.mark.parametrize("world", [1, 2, 3])
def test_graph_shares_equal_the_whole_batch(gpu, world):
    vo, eo, rp, cl, deg = ragged_arrays()
    whole = np.empty(int(vo[-1]), np.float32)
    with GraphBatch(vo, eo, rp, cl) as bt:
        st = bt.page_rank(deg, whole, D, 1e-6, 200)
    assert st.converged_graphs == len(vo) - 1
    b = S.graph_bounds(vo, eo, world)
    for q in range(world):
        lo, hi = int(b[q]), int(b[q + 1])
        if hi == lo:
            continue
        v0, v1 = int(vo[lo]), int(vo[hi])
        part = np.empty(v1 - v0, np.float32)
        with GraphBatch(*S.batch_slice(vo, eo, rp, cl, lo, hi)) as bt:
            sq = bt.page_rank(np.ascontiguousarray(deg[v0:v1]), part, D, 1e-6, 200)
        assert np.array_equal(part.view(np.uint32), whole[v0:v1].view(np.uint32)), (world, q)
        assert np.array_equal(sq.graph_iterations, st.graph_iterations[lo:hi])


def test_distributed_entry_points_on_one_rank(gpu, ppr_case, nccl_one_rank):
    g, deg, seeds = ppr_case
    whole, st = whole_ppr(g, deg, seeds)
    dev = torch.device("cuda", 0)
    deg_d = torch.from_numpy(deg.view(np.int32)).to(dev)
    with Graph(torch.from_numpy(g.row_ptr.view(np.int32)).to(dev), torch.from_numpy(g.col.view(np.int32)).to(dev)) as h:
        scores, sst = S.ppr_batched(h, deg_d, seeds, D, 1e-6, 100, group=nccl_one_rank)
    assert np.array_equal(scores.cpu().numpy().view(np.uint32), whole.view(np.uint32))
    assert sst.columns == (0, len(seeds)) and sst.iterations == st.iterations and sst.all_converged
    assert np.array_equal(sst.col_iterations, st.col_iterations)

    vo, eo, rp, cl, dg = ragged_arrays()
    ref = np.empty(int(vo[-1]), np.float32)
    with GraphBatch(vo, eo, rp, cl) as bt:
        bt.page_rank(dg, ref, D, 1e-6, 200)
    sb = S.ShardedBatch(vo, eo, torch.from_numpy(rp.view(np.int32)).to(dev), torch.from_numpy(cl.view(np.int32)).to(dev),
                        group=nccl_one_rank)
    try:
        v0, v1 = sb.vertex_range
        local = torch.empty(v1 - v0, dtype=torch.float32, device=dev)
        sb.page_rank(torch.from_numpy(dg[v0:v1].view(np.int32)).to(dev), local, D, 1e-6, 200)
        got = sb.gather(local)
    finally:
        sb.release()
    assert np.array_equal(got.cpu().numpy().view(np.uint32), ref.view(np.uint32))
