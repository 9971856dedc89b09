"""Weighted SpMV through the PageRank engine (nwgpu_spmv): y[i] = sum over row
i's entries of w[k] * x[col[k]], the reference's SpMV kernel
(bench/abstraction_penalty/spmv.cpp:52-62: y[i] += x[idx[j]] * dat[j] from
y = 0). The reference sums each row serially in FP32; the engine sums in its
own fixed order, so the bar is FP32 accuracy: each y[i] within 1e-6 relative
of the FP64 sum of |terms|, and bitwise reproducible."""
import numpy as np
import pytest

from nwgraph_b200 import Graph, NwgpuError, graphs as G
from nwgraph_b200 import _native as N

pytestmark = pytest.mark.gpu


def spmv64(rp, cl, w, x):
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp.astype(np.int64)))
    t = w.astype(np.float64) * x.astype(np.float64)[cl]
    return np.bincount(rows, weights=t, minlength=len(rp) - 1), np.bincount(rows, weights=np.abs(t), minlength=len(rp) - 1)


def serial_f32(rp, cl, w, x):
    """The reference loop on one thread, in FP32 (products rounded, then added)."""
    y = np.zeros(len(rp) - 1, np.float32)
    lens = np.diff(rp.astype(np.int64))
    for k in range(int(lens.max())):
        r = np.nonzero(lens > k)[0]
        y[r] = (y[r] + (x[cl[rp[r] + k]] * w[rp[r] + k]).astype(np.float32)).astype(np.float32)
    return y


@pytest.mark.parametrize("graph", ["rmat16", "directed", "grid"])
def test_spmv_matches_fp64_and_reference_loop(gpu, graph):
    rng = np.random.default_rng(4)
    if graph == "rmat16":
        g = G.rmat(16, 16, 2)
    elif graph == "grid":
        g = G.grid(40000)
    else:
        src = rng.integers(0, 30000, 300000)
        dst = (rng.pareto(1.2, 300000) * 20).astype(np.int64) % 30000
        g = G.from_edges(src, dst, 30000)
    w = G.edge_weights(g.nnz, seed=9)
    x = rng.standard_normal(g.n).astype(np.float32)
    with Graph(g.row_ptr, g.col, weights=w) as h:
        y = np.empty(g.n, np.float32)
        h.spmv(x, y)
        y2 = np.empty(g.n, np.float32)
        h.spmv(x, y2)
    exact, mag = spmv64(g.row_ptr, g.col, w, x)
    assert np.all(np.abs(y - exact) <= 1e-6 * mag + 1e-30)
    ser = serial_f32(g.row_ptr, g.col, w, x)
    assert np.all(np.abs(y.astype(np.float64) - ser) <= 2e-6 * mag + 1e-30)
    assert np.array_equal(y.view(np.uint32), y2.view(np.uint32))


def test_spmv_device_pointers_and_errors(gpu):
    import torch
    g = G.rmat(12, 16, 3)
    w = G.edge_weights(g.nnz, seed=1)
    x = np.random.default_rng(0).standard_normal(g.n).astype(np.float32)
    with Graph(g.row_ptr, g.col, weights=w) as h:
        yh = np.empty(g.n, np.float32)
        h.spmv(x, yh)
        yd = torch.empty(g.n, dtype=torch.float32, device="cuda")
        h.spmv(torch.from_numpy(x).cuda(), yd)
        assert np.array_equal(yd.cpu().numpy(), yh)
    with Graph(g.row_ptr, g.col) as h:  # no weights
        with pytest.raises(NwgpuError) as ei:
            h.spmv(x, np.empty(g.n, np.float32))
        assert ei.value.status == N.ERR_UNSUPPORTED
