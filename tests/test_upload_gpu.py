"""The streamed build of a host CSR (nwgpu_graph_create with host pointers):
the row pointers are uploaded and checked first, the column ids follow in
merge-path chunks while the rows are sorted, and each chunk's entries are
placed in the relabelled CSR as it arrives. NWGPU_UPLOAD_CHUNK_ENTRIES makes
the chunks small here, so rows cross chunk boundaries and chunks hold only
empty rows. The result must be the relabelled CSR of the one-piece path
(device pointers): equal launch plans and bitwise-equal ranks; invalid input
is rejected with the one-piece path's errors.
"""
import numpy as np
import pytest
import torch

from nwgraph_b200 import Graph, NwgpuError, graphs as G
from nwgraph_b200 import _native as N

pytestmark = pytest.mark.gpu


def directed_with_gaps(n=30000, m=300000, seed=5):
    """Power-law targets, sources only in [1000, n - 1000): empty rows at both ends."""
    rng = np.random.default_rng(seed)
    src = rng.integers(1000, n - 1000, m)
    dst = (rng.pareto(1.2, m) * 20).astype(np.int64) % n
    keep = src != dst
    return G.from_edges(dst[keep], src[keep], n)


def one_big_row(n=5000):
    src = np.zeros(n - 1, np.int64)
    dst = np.arange(1, n)
    return G.from_edges(np.concatenate([src, dst]), np.concatenate([dst, src]), n)


GRAPHS = {"rmat14": lambda: G.rmat(14, 16, 3), "grid": lambda: G.grid(40000), "gaps": directed_with_gaps,
          "hub": one_big_row}


def ranks(h, deg, iters=20):
    out = np.empty(h.n, np.float32)
    h.page_rank(deg, out, 0.85, 0.0, iters)
    return out


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("chunk", [1, 777, 65536])
def test_streamed_build_equals_one_piece(gpu, monkeypatch, name, chunk):
    g = GRAPHS[name]()
    deg = g.out_degree()
    dev = torch.device("cuda", 0)
    with Graph(torch.from_numpy(g.row_ptr.view(np.int32)).to(dev), torch.from_numpy(g.col.view(np.int32)).to(dev)) as h:
        want, want_info = ranks(h, deg), h.info()
    monkeypatch.setenv("NWGPU_UPLOAD_CHUNK_ENTRIES", str(chunk))
    with Graph(g.row_ptr, g.col) as h:
        got, info = ranks(h, deg), h.info()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    for k in ("binned", "sweep_grid", "num_tiles", "hub_smem_ids"):
        assert info[k] == want_info[k], k


@pytest.mark.parametrize("chunk", [1, 2])
def test_streamed_build_rejects_invalid_input(gpu, monkeypatch, chunk):
    monkeypatch.setenv("NWGPU_UPLOAD_CHUNK_ENTRIES", str(chunk))
    with pytest.raises(NwgpuError) as ei:  # a column id >= n, found while the entries are placed
        Graph(np.array([0, 2, 3, 5], np.uint32), np.array([1, 2, 7, 0, 1], np.uint32))
    assert ei.value.status == N.ERR_INVALID_GRAPH and "col" in str(ei.value)
    with pytest.raises(NwgpuError) as ei:  # decreasing row pointers, found before any entry is placed
        Graph(np.array([0, 3, 1, 5], np.uint32), np.array([1, 0, 2, 0, 1], np.uint32))
    assert ei.value.status == N.ERR_INVALID_GRAPH and "decreases" in str(ei.value)
    with pytest.raises(NwgpuError) as ei:  # row_ptr[n] != nnz
        Graph(np.array([0, 1, 2, 3], np.uint32), np.array([1, 0, 0, 2, 1], np.uint32), nnz=5)
    assert ei.value.status == N.ERR_INVALID_GRAPH
    g = G.rmat(10, 8, 2)  # the handle after a rejected one still works
    with Graph(g.row_ptr, g.col) as h:
        assert np.isfinite(ranks(h, g.out_degree(), 3)).all()
