"""Row-sharded solve (nwgraph_b200/shard.py) on CPU: the partition, the padded
all-gather layout, the exchange protocol and the stopping rule, with the
CPU stand-in of a shard (tests/oracle_shard.py) in place of the GPU kernels.

* one process holding 1..4 shards (LocalExchange) gives the same ranks bit
  for bit as one shard, and one shard matches page_rank_v10 (the oracle's
  jacobi_f32, pinned to the reference in test_oracle.py);
* two gloo ranks under torch.distributed.run (DistExchange, the launcher
  bench.py uses) give the one-process result on both ranks;
* batches shard with no exchange per sweep: personalised columns split
  evenly, ragged batches by whole graphs balanced by rows plus entries; three
  gloo ranks (tests/batch_shard_worker.py, oracle solves in place of the GPU)
  assemble the whole batch's result bit for bit.
"""
import os
import sys

import numpy as np
import pytest
import torch

import oracle as O
from nwgraph_b200 import graphs as G, shard as S

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from oracle_shard import OracleShard  # noqa: E402
from test_multirank import torchrun  # noqa: E402


def solve_local(g, world, thr, iters):
    bounds, stride = S.shard_bounds(g.row_ptr, world)
    shards = [OracleShard(g.row_ptr, g.col, world, q, bounds, stride) for q in range(world)]
    out = torch.zeros(g.n, dtype=torch.float32)
    st = S.run(shards, S.LocalExchange(), g.out_degree(), out, 0.85, thr, iters, device="cpu")
    return out.numpy().copy(), st


@pytest.mark.parametrize("world", [1, 2, 3, 5, 8])
def test_bounds_cover_rows_and_balance_work(world):
    g = G.rmat(12, 16, 1)
    bounds, stride = S.shard_bounds(g.row_ptr, world)
    assert bounds[0] == 0 and bounds[-1] == g.n and np.all(np.diff(bounds.astype(np.int64)) >= 0)
    assert stride % 4 == 0 and stride >= np.diff(bounds.astype(np.int64)).max()
    lens = np.sort(np.diff(g.row_ptr.astype(np.int64)))[::-1]
    rp = np.concatenate([[0], np.cumsum(lens)])
    work = [(rp[b] + b) - (rp[a] + a) for a, b in zip(bounds[:-1].astype(np.int64), bounds[1:].astype(np.int64))]
    # every range is within one row of an equal share of rows + entries
    assert max(work) - (g.n + g.nnz) / world <= lens[0] + 1


def test_more_ranks_than_rows_leaves_empty_ranges():
    g = G.grid(4)
    bounds, stride = S.shard_bounds(g.row_ptr, 8)
    assert bounds[-1] == 4 and stride == 4
    out, st = solve_local(g, 8, 0.0, 5)
    ref, _, _ = O.jacobi_f32(g.row_ptr, g.col, g.out_degree(), 0.85, 0.0, 5)
    assert np.abs(out - ref).max() <= 1e-6


@pytest.mark.parametrize("world", [2, 3, 4])
def test_local_shards_equal_one_shard(world):
    g = G.rmat(10, 16, 3)
    one, st1 = solve_local(g, 1, 0.0, 15)
    many, stw = solve_local(g, world, 0.0, 15)
    assert np.array_equal(one.view(np.uint32), many.view(np.uint32))
    assert st1.iterations == stw.iterations == 15
    assert np.allclose(st1.errors, stw.errors, rtol=1e-12, atol=0)


def test_one_shard_matches_page_rank_v10():
    g = G.rmat(10, 16, 3)
    deg = g.out_degree()
    out, st = solve_local(g, 1, 1e-6, 200)
    ref, it, errs = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 1e-6, 200)
    assert st.converged and st.iterations == it
    assert np.abs(out.astype(np.float64) - ref).max() <= 1e-6
    assert np.allclose(st.errors, errs, rtol=1e-4, atol=2.5e-7)


def test_two_gloo_ranks_match_one_process(tmp_path):
    res = torchrun([os.path.join("tests", "shard_worker.py"), str(tmp_path), "1e-6", "200"])
    assert res.returncode == 0, res.stderr[-3000:]
    g = G.rmat(10, 16, 3)
    local, st = solve_local(g, 2, 1e-6, 200)
    for r in range(2):
        z = np.load(tmp_path / f"rank{r}.npz")
        assert int(z["iterations"]) == st.iterations
        assert np.array_equal(z["ranks"].view(np.uint32), local.view(np.uint32))
        assert np.allclose(z["errors"], st.errors, rtol=1e-12, atol=0)


@pytest.mark.parametrize("count,world", [(0, 1), (0, 3), (7, 3), (64, 8), (5, 8), (1000, 7)])
def test_even_bounds(count, world):
    b = S.even_bounds(count, world)
    sizes = np.diff(b)
    assert b[0] == 0 and b[-1] == count and len(b) == world + 1
    assert sizes.min() >= 0 and sizes.max() - sizes.min() <= 1 and np.all(np.diff(sizes) <= 0)


@pytest.mark.parametrize("world", [1, 2, 3, 4, 9])
def test_weighted_bounds_cut_at_the_nearest_boundary(world):
    w = np.random.default_rng(world).integers(1, 100, 40)
    b = S.weighted_bounds(w, world)
    ends = np.concatenate([[0], np.cumsum(w)])
    assert b[0] == 0 and b[-1] == len(w) and np.all(np.diff(b) >= 0)
    for q in range(1, world):
        t = q * ends[-1] / world
        assert abs(ends[b[q]] - t) == np.abs(ends - t).min()
    assert np.array_equal(S.weighted_bounds([], 3), [0, 0, 0, 0])


def test_batch_slice_keeps_each_graph():
    graphs = [G.rmat(6, 4, s) for s in range(5)] + [G.grid(49)]
    vo = np.concatenate([[0], np.cumsum([g.n for g in graphs])]).astype(np.uint64)
    eo = np.concatenate([[0], np.cumsum([g.nnz for g in graphs])]).astype(np.uint64)
    rp = np.concatenate([g.row_ptr for g in graphs])
    cl = np.concatenate([g.col for g in graphs])
    for lo, hi in [(0, 6), (1, 4), (5, 6), (3, 3)]:
        svo, seo, srp, scl = S.batch_slice(vo, eo, rp, cl, lo, hi)
        assert svo[0] == 0 and seo[0] == 0 and len(srp) == int(svo[-1]) + hi - lo and len(scl) == int(seo[-1])
        for j, g in enumerate(graphs[lo:hi]):
            assert np.array_equal(srp[int(svo[j]) + j:int(svo[j + 1]) + j + 1], g.row_ptr)
            assert np.array_equal(scl[int(seo[j]):int(seo[j + 1])], g.col)
    b = S.graph_bounds(vo, eo, 3)
    assert b[0] == 0 and b[-1] == len(graphs)


def test_three_gloo_ranks_assemble_the_whole_batches(tmp_path):
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import batch_shard_worker as W
    res = torchrun([os.path.join("tests", "batch_shard_worker.py"), str(tmp_path)], nproc=3)
    assert res.returncode == 0, res.stderr[-3000:]
    g, deg, seeds = W.ppr_case()
    whole = np.stack([O.ppr_jacobi_f32(g.row_ptr, g.col, deg, int(s), W.D, W.THR, W.ITERS)[0] for s in seeds], 1)
    its = [O.ppr_jacobi_f32(g.row_ptr, g.col, deg, int(s), W.D, W.THR, W.ITERS)[1] for s in seeds]
    graphs, vo, eo, _, _ = W.ragged_case()
    ragged = np.concatenate([O.jacobi_f32(x.row_ptr, x.col, x.out_degree(), W.D, W.THR, 200)[0] for x in graphs])
    b = S.even_bounds(len(seeds), 3)
    for r in range(3):
        z = np.load(tmp_path / f"rank{r}.npz")
        assert np.array_equal(z["scores"].view(np.uint32), whole.view(np.uint32))
        assert tuple(z["columns"]) == (b[r], b[r + 1])
        assert np.array_equal(z["block"].view(np.uint32), whole[:, b[r]:b[r + 1]].view(np.uint32))
        assert np.array_equal(z["col_iterations"], its) and int(z["iterations"]) == max(its)
        assert bool(z["all_converged"]) and np.all(z["col_converged"]) and float(z["device_ms"]) == 3.0
        assert np.array_equal(z["ragged"].view(np.uint32), ragged.view(np.uint32))
        assert np.array_equal(z["graph_bounds"], S.graph_bounds(vo, eo, 3))
