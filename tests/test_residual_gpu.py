"""Residual-push PageRank (nwgpu_pr_residual_run) against page_rank_v13
(experimental/algorithms/page_rank.hpp:552-625), through the oracle's
restatement oracle.residual_f32, which equals the compiled reference bit for
bit (test_oracle.py).

The engine sums each vertex's incoming deltas in its kernel's order, not
serially, so sums differ in their last bits. With threshold 0 every positive
residual pushes and the runs stay in step: ranks agree to 1e-6 relative (they
are O(1): v13 does not normalise) and the push counts per iteration agree
exactly. With a real threshold a residual within rounding of it may push in
one run and not in the other (v13 then drops it), so ranks may differ by a
few times the threshold and the iteration count by one.
"""
import numpy as np
import pytest

import oracle as O
from nwgraph_b200 import Graph, NwgpuError, graphs as G
from nwgraph_b200 import _native as N

pytestmark = pytest.mark.gpu


def directed(n=20000, m=200000, seed=3):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, n, m)
    dst = (rng.pareto(1.3, m) * 30).astype(np.int64) % n
    keep = (src < n - 50) & (src != dst)  # the last 50 vertices have no out-edges
    return G.from_edges(src[keep], dst[keep], n)


def residual_f64(g, deg, d, thr, iters):
    """page_rank_v13's iteration in FP64 (the exact arithmetic the FP32 runs approximate)."""
    rows = np.repeat(np.arange(g.n), np.diff(g.row_ptr.astype(np.int64)))
    pr = np.zeros(g.n)
    res = np.full(g.n, 1.0 - d)
    for _ in range(iters):
        push = res > thr
        moved = push & (deg > 0)
        pr[push] += res[push]
        delta = np.where(moved, res * d / np.maximum(deg, 1), 0.0)
        s = np.bincount(rows, weights=delta[g.col], minlength=g.n)
        res = np.where(s > 0, s, 0.0)
        if not moved.any():
            break
    return pr


def close_or_more_accurate(gpu, ref, exact, rel=1e-6):
    """Within rel of the reference, or, where the reference's serial FP32 sums
    are themselves further than rel from FP64 (hub rows), at least as close to
    FP64 as the reference."""
    scale = np.maximum(np.abs(exact), 1e-3)
    if np.all(np.abs(gpu.astype(np.float64) - ref) <= rel * scale):
        return True
    e_ref = np.abs(ref.astype(np.float64) - exact) / scale
    e_gpu = np.abs(gpu.astype(np.float64) - exact) / scale
    return e_ref.max() > rel and e_gpu.max() <= 1.01 * e_ref.max() and e_gpu.sum() <= 1.01 * e_ref.sum()


GRAPHS = {"rmat14": lambda: G.rmat(14, 16, 4), "grid": lambda: G.grid(30000), "directed": directed}


def run(g, deg, thr, iters, launch="graph"):
    with Graph(g.row_ptr, g.col) as h:
        out = np.empty(g.n, np.float32)
        st = h.page_rank_residual(deg, out, 0.85, thr, iters, launch=launch, record_errors=True)
    return out, st


@pytest.mark.parametrize("name", list(GRAPHS))
def test_every_residual_pushes(gpu, name):
    g = GRAPHS[name]()
    deg = g.out_degree()
    out, st = run(g, deg, 0.0, 12)
    ref, it, cnt = O.residual_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 12)
    assert st.iterations == it == 12
    assert np.allclose(st.errors, cnt, rtol=0, atol=0)
    assert close_or_more_accurate(out, ref, residual_f64(g, deg, 0.85, 0.0, 12))
    out2, _ = run(g, deg, 0.0, 12, launch="stream")
    assert np.array_equal(out.view(np.uint32), out2.view(np.uint32))


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("thr", [1e-4, 1e-3])
def test_threshold_runs(gpu, name, thr):
    g = GRAPHS[name]()
    deg = g.out_degree()
    out, st = run(g, deg, thr, 200)
    ref, it, cnt = O.residual_f32(g.row_ptr, g.col, deg, 0.85, thr, 200)
    assert st.converged and abs(st.iterations - it) <= 1
    assert st.errors[0] == cnt[0]
    assert np.all(np.abs(out.astype(np.float64) - ref) <= 4 * thr + 1e-5 * np.abs(ref))


def test_edge_cases(gpu):
    g = G.rmat(10, 16, 1)
    deg = g.out_degree()
    out, st = run(g, deg, 1e-4, 0)  # no iteration: ranks stay 0
    assert st.iterations == 0 and np.all(out == 0)
    out, st = run(g, deg, 1e-4, 1)  # one iteration: every vertex pushed 1 - d (d the FP32 damping, :567)
    assert st.iterations == 1 and np.all(out == np.float32(1.0 - np.float64(np.float32(0.85))))
    out, st = run(g, deg, 0.5, 10)  # 1 - d below the threshold: nothing pushes
    assert st.iterations == 1 and st.converged and np.all(out == 0)
    with Graph(g.row_ptr, g.col, relabel=False) as h:
        with pytest.raises(NwgpuError) as ei:
            h.page_rank_residual(deg, np.empty(g.n, np.float32))
        assert ei.value.status == N.ERR_UNSUPPORTED
