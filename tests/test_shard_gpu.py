"""Row-sharded solve on the GPU (nwgpu_shard_* through nwgraph_b200.shard).

Each row is summed by the same binned-sweep code whichever shard owns it, so
at a fixed sweep count the sharded ranks equal the single-GPU engine's
(nwgpu_pr_run) bit for bit. Several shards run here in one process on one GPU
(LocalExchange: their kernels never wait on one another; the slices are
copied into the padded layout between sweeps); the exchange over
torch.distributed is covered on CPU by tests/test_shard.py with two gloo ranks,
and here by ShardedGraph over a one-rank NCCL group (all_gather_into_tensor and
all_reduce on device buffers).
"""
import numpy as np
import pytest

import oracle as O
from nwgraph_b200 import Graph, NwgpuError, graphs as G, shard as S
from nwgraph_b200 import _native as N

pytestmark = pytest.mark.gpu


def sharded(g, deg, world, thr, iters, device_inputs=False):
    import torch
    dev = torch.device("cuda")
    bounds, stride = S.shard_bounds(g.row_ptr, world)
    rp, cl, dg = g.row_ptr, g.col, deg
    if device_inputs:
        rp = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
        cl = torch.from_numpy(g.col.view(np.int32)).to(dev)
        dg = torch.from_numpy(deg.view(np.int32)).to(dev)
    shards = [S.GpuShard(rp, cl, world, q, bounds, stride) for q in range(world)]
    out = torch.empty(g.n, dtype=torch.float32, device=dev)
    st = S.run(shards, S.LocalExchange(), dg, out, 0.85, thr, iters, device=dev)
    for s in shards:
        s.release()
    return out.cpu().numpy(), st


def single(g, deg, thr, iters):
    with Graph(g.row_ptr, g.col) as h:
        out = np.empty(g.n, np.float32)
        st = h.page_rank(deg, out, 0.85, thr, iters, record_errors=True)
    return out, st


@pytest.mark.parametrize("scale", [14, 18])
def test_shards_equal_single_gpu_engine(gpu, scale):
    g = G.rmat(scale, 16, 7)
    deg = g.out_degree()
    ref, st_ref = single(g, deg, 0.0, 20)
    for world in (1, 2, 3, 4):
        out, st = sharded(g, deg, world, 0.0, 20, device_inputs=(world == 3))
        assert st.iterations == 20
        assert np.array_equal(out.view(np.uint32), ref.view(np.uint32)), world
        assert np.allclose(st.errors, st_ref.errors, rtol=1e-9, atol=0), world


def test_threshold_run_matches_page_rank_v10(gpu):
    g = G.rmat(16, 16, 3)
    deg = g.out_degree()
    out, st = sharded(g, deg, 3, 1e-4, 100)
    ref, it, errs = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 1e-4, 100)
    assert st.converged and st.iterations == it
    d = np.abs(out.astype(np.float64) - ref)
    assert d.max() <= 1e-6 and d.sum() <= 1e-5
    assert np.allclose(st.errors, errs, rtol=1e-4, atol=1e-6)


def test_more_ranks_than_rows(gpu):
    g = G.grid(9)
    deg = g.out_degree()
    ref, _ = single(g, deg, 0.0, 10)
    out, _ = sharded(g, deg, 6, 0.0, 10)
    assert np.abs(out - ref).max() <= 1e-7


def test_invalid_bounds(gpu):
    g = G.rmat(10, 16, 1)
    bounds, stride = S.shard_bounds(g.row_ptr, 2)
    bad = bounds.copy()
    bad[-1] -= 1
    with pytest.raises(NwgpuError) as ei:
        S.GpuShard(g.row_ptr, g.col, 2, 0, bad, stride)
    assert ei.value.status == N.ERR_INVALID_ARG
    with pytest.raises(NwgpuError) as ei:
        S.GpuShard(g.row_ptr, g.col, 2, 0, bounds, stride - 2)
    assert ei.value.status == N.ERR_INVALID_ARG
    with pytest.raises(NwgpuError):
        S.GpuShard(g.row_ptr, g.col, 2, 2, bounds, stride)


def test_sharded_graph_over_nccl_one_rank(gpu, nccl_one_rank):
    import torch
    g = G.rmat(16, 16, 4)
    deg = g.out_degree()
    want, _ = single(g, deg, 0.0, 20)
    dev = torch.device("cuda", 0)
    sg = S.ShardedGraph(torch.from_numpy(g.row_ptr.view(np.int32)).to(dev),
                        torch.from_numpy(g.col.view(np.int32)).to(dev), group=nccl_one_rank)
    try:
        out = torch.empty(g.n, dtype=torch.float32, device=dev)
        st = sg.page_rank(torch.from_numpy(deg.view(np.int32)).to(dev), out, 0.85, 0.0, 20)
    finally:
        sg.release()
    assert st.iterations == 20 and len(st.errors) == 20
    assert np.array_equal(out.cpu().numpy().view(np.uint32), want.view(np.uint32))
