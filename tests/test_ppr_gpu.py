"""Personalised PageRank on the GPU: single-seed solves and the batched SpMM.

No counterpart in the reference; the oracles are the FP32 restatement of
page_rank_v10 with a one-hot teleport (oracle.ppr_jacobi_f32, same sweep and
stopping rule) and the FP64 power iteration (oracle.pr_f64 with a teleport).
"""
import numpy as np
import pytest

import oracle as O
from nwgraph_b200 import Graph, NwgpuError, graphs as G
from nwgraph_b200 import _native as N

pytestmark = pytest.mark.gpu

MAX_ABS = 1e-6
L1 = 1e-5


def close(a, b, max_abs=MAX_ABS, l1=L1):
    d = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))
    assert d.max() <= max_abs, f"max-abs {d.max():.3e}"
    assert d.sum() <= l1, f"L1 {d.sum():.3e}"


@pytest.fixture(scope="module")
def rmat13():
    g = G.rmat(13, 16, 5)
    return g, g.out_degree()


def test_single_seed_matches_restatement(gpu, rmat13):
    g, deg = rmat13
    seeds = G.random_sources(deg, 4, seed=7)
    with Graph(g.row_ptr, g.col) as h:
        for s in seeds:
            out = np.empty(g.n, np.float32)
            st = h.ppr(deg, int(s), out, 0.85, 0.0, 25, record_errors=True)
            ref, it, errs = O.ppr_jacobi_f32(g.row_ptr, g.col, deg, int(s), 0.85, 0.0, 25)
            assert st.iterations == 25
            close(out, ref)
            assert np.allclose(st.errors, errs, rtol=1e-4, atol=1e-6)
            # threshold run: at 1e-6 the L1 change of a sweep is within a few percent of the FP32
            # rounding noise of O(1) ranks, so the stopping sweep may differ by one at a near-tie
            st = h.ppr(deg, int(s), out, 0.85, 1e-6, 200)
            ref, it, _ = O.ppr_jacobi_f32(g.row_ptr, g.col, deg, int(s), 0.85, 1e-6, 200)
            assert abs(st.iterations - it) <= 1 and st.converged
            close(out, ref)


def test_single_seed_vs_fp64(gpu, rmat13):
    g, deg = rmat13
    s = int(G.random_sources(deg, 1, seed=3)[0])
    t = np.zeros(g.n)
    t[s] = 1.0
    r64, _, _ = O.pr_f64(g.row_ptr, g.col, teleport=t, tol=1e-15)
    with Graph(g.row_ptr, g.col) as h:
        out = np.empty(g.n, np.float32)
        h.ppr(deg, s, out, 0.85, 1e-7, 500)
    assert np.abs(out - r64).max() < 2e-6
    assert abs(float(out.astype(np.float64).sum()) - 1.0) < 1e-4  # symmetric graph: no mass leaks from the seed


@pytest.mark.parametrize("k", [1, 5, 32, 40, 64, 100])
def test_batched_matches_single(gpu, rmat13, k):
    g, deg = rmat13
    seeds = G.random_sources(deg, k, seed=11)
    with Graph(g.row_ptr, g.col) as h:
        out = np.empty((g.n, k), np.float32)
        st = h.ppr_batched(deg, seeds, out, 0.85, 1e-6, 200)
        assert st.all_converged and st.col_converged.all()
        for c in range(0, k, max(1, k // 6)):
            ref, it, _ = O.ppr_jacobi_f32(g.row_ptr, g.col, deg, int(seeds[c]), 0.85, 1e-6, 200)
            close(out[:, c], ref)
            # per-column stopping rule (sums of n FP32 differences: allow one sweep of slack at a tie)
            assert abs(int(st.col_iterations[c]) - it) <= 1
        assert st.iterations == int(st.col_iterations.max())


def test_batched_fixed_sweeps_exact_columns(gpu, rmat13):
    g, deg = rmat13
    seeds = G.random_sources(deg, 64, seed=2)
    with Graph(g.row_ptr, g.col) as h:
        out = np.empty((g.n, 64), np.float32)
        st = h.ppr_batched(deg, seeds, out, 0.85, 0.0, 15)
        assert st.iterations == 15 and not st.all_converged
        assert (st.col_iterations == 15).all()
        for c in (0, 17, 63):
            ref, _, _ = O.ppr_jacobi_f32(g.row_ptr, g.col, deg, int(seeds[c]), 0.85, 0.0, 15)
            close(out[:, c], ref)


def test_batched_hubs_and_duplicate_seeds(gpu):
    # hub rows spanning many warp tiles, two columns with the same seed
    n = 30_001
    s = np.zeros(n - 1, np.uint32)
    d = np.arange(1, n, dtype=np.uint32)
    g = G.from_edges(s, d, n, symmetrize=True)
    deg = g.out_degree()
    seeds = np.array([0, 5, 5, 29_000], np.uint32)
    with Graph(g.row_ptr, g.col) as h:
        out = np.empty((n, 4), np.float32)
        h.ppr_batched(deg, seeds, out, 0.85, 0.0, 12)
    assert np.array_equal(out[:, 1], out[:, 2])
    for c in range(4):
        ref, _, _ = O.ppr_jacobi_f32(g.row_ptr, g.col, deg, int(seeds[c]), 0.85, 0.0, 12)
        exact, _, _ = O.pr_f64(g.row_ptr, g.col, teleport=np.eye(1, n, int(seeds[c]))[0], tol=0.0, max_iters=12)
        e_gpu = np.abs(out[:, c] - exact).max()
        e_ref = np.abs(ref - exact).max()
        assert np.abs(out[:, c] - ref).max() <= 1e-6 or e_gpu <= e_ref * 1.01 + 1e-9


def test_batched_device_pointers(gpu, rmat13):
    import torch
    g, deg = rmat13
    seeds = G.random_sources(deg, 64, seed=4)
    dev = torch.device("cuda")
    with Graph(g.row_ptr, g.col) as h:
        out_h = np.empty((g.n, 64), np.float32)
        h.ppr_batched(deg, seeds, out_h, 0.85, 1e-6, 200)
        out_d = torch.empty((g.n, 64), dtype=torch.float32, device=dev)
        h.ppr_batched(torch.from_numpy(deg.view(np.int32)).to(dev), seeds, out_d, 0.85, 1e-6, 200, launch="stream")
        torch.cuda.synchronize()
    assert np.array_equal(out_d.cpu().numpy(), out_h)


def test_ppr_bad_arguments(gpu, rmat13):
    g, deg = rmat13
    with Graph(g.row_ptr, g.col) as h:
        with pytest.raises(NwgpuError) as ei:
            h.ppr(deg, g.n + 3, np.empty(g.n, np.float32))
        assert ei.value.status == N.ERR_INVALID_ARG
        with pytest.raises(NwgpuError):
            h.ppr_batched(deg, np.array([g.n], np.uint32), np.empty((g.n, 1), np.float32))
        with pytest.raises(NwgpuError):
            h.ppr_batched(deg, np.zeros(129, np.uint32), np.empty((g.n, 129), np.float32))
