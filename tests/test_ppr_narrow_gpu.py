"""Narrowing of the batched personalised solve (nwgpu_ppr_batched).

Once at most K/2 of a batch's K padded columns still run, the solve moves the
running columns into an n x K/2 layout and goes on with the narrower kernels
(128 -> 64 -> 32). Every column is summed in the same order at every width,
so a batch that narrows must give, bit for bit and with the same sweep
counts, what the same seeds give in batches of at most 32 columns, which
never narrow.
"""
import numpy as np
import pytest

from nwgraph_b200 import Graph, graphs as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graph():
    g = G.rmat(14, 16, 5)
    return g, g.out_degree()


def solve(h, deg, seeds, iters=100, launch="graph"):
    out = np.empty((len(deg), len(seeds)), np.float32)
    st = h.ppr_batched(deg, seeds, out, 0.85, 1e-6, iters, launch=launch)
    return out, st


@pytest.mark.parametrize("k", [64, 100, 128])
@pytest.mark.parametrize("iters", [100, 15])
def test_narrowed_batch_equals_32_column_batches(gpu, graph, k, iters):
    g, deg = graph
    seeds = G.random_sources(deg, k, seed=3)
    with Graph(g.row_ptr, g.col) as h:
        whole, st = solve(h, deg, seeds, iters)
        if iters == 100:  # the columns stop at different sweeps, so the loop narrowed
            assert st.all_converged and st.col_iterations.min() < st.iterations
        for c0 in range(0, k, 32):
            part, sp = solve(h, deg, seeds[c0:c0 + 32], iters)
            assert np.array_equal(part.view(np.uint32), whole[:, c0:c0 + 32].view(np.uint32)), c0
            assert np.array_equal(sp.col_iterations, st.col_iterations[c0:c0 + 32])
            assert np.array_equal(sp.col_converged, st.col_converged[c0:c0 + 32])
        again, s2 = solve(h, deg, seeds, iters, launch="stream")
    assert np.array_equal(again.view(np.uint32), whole.view(np.uint32)) and s2.iterations == st.iterations


def test_abort_in_a_narrowed_phase(gpu):
    """39 seeds on isolated vertices stop exactly at their second sweep; the
    40th, on a bipartite grid with d = 1, oscillates and never stops. The loop
    narrows right away and then runs in its narrowed phase until aborted."""
    import threading
    import time

    from nwgraph_b200 import NwgpuError
    from nwgraph_b200 import _native as N
    grid = G.grid(10000)
    iso = 39
    rp = np.concatenate([grid.row_ptr, np.full(iso, grid.row_ptr[-1], np.uint32)])
    n = len(rp) - 1
    deg = np.concatenate([grid.out_degree(), np.zeros(iso, np.uint32)])
    seeds = np.concatenate([np.arange(grid.n, n), [grid.n // 2]]).astype(np.uint32)
    out = np.empty((n, len(seeds)), np.float32)
    with Graph(rp, grid.col) as h:
        t = threading.Timer(0.5, h.abort)
        t.start()
        t0 = time.time()
        with pytest.raises(NwgpuError) as ei:
            h.ppr_batched(deg, seeds, out, 1.0, 1e-30, 2_000_000)
        t.join()
        assert ei.value.status == N.ERR_ABORTED
        assert time.time() - t0 < 30
        st = h.ppr_batched(deg, seeds[:4], np.empty((n, 4), np.float32), 0.85, 1e-6, 100)  # still usable
        assert st.all_converged
