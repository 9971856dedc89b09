"""Weighted PageRank and the implicit adjoint (nwgpu_wpr_run, nwgpu_pr_vjp).

No counterpart in the reference (its page_rank is unweighted); the oracles
are the FP64 restatements oracle.pr_f64 (weighted, out-normalised, with a
teleport vector, leak semantics) and oracle.vjp_f64 (the adjoint of the fixed
point and the gradients), plus FP64 central finite differences of
L = c . r(w, t) with step 1e-3 on raw edge weights (re-normalised by the
solve) and teleport entries. Bars: forward within 1e-6 max-abs of FP64,
gradients within 1e-4 relative of the FP64 oracle and of the finite
differences.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from nwgraph_b200 import Graph, NwgpuError, graphs as G
from nwgraph_b200 import _native as N

pytestmark = pytest.mark.gpu

D = 0.85


@pytest.fixture(scope="module")
def wgraph():
    g = G.rmat(13, 16, 21)
    w = G.edge_weights(g.nnz, seed=1234)
    rng = np.random.default_rng(99)
    c = rng.standard_normal(g.n).astype(np.float32)
    t = rng.uniform(0.5, 1.5, g.n)
    t = (t / t.sum()).astype(np.float32)
    return g, w, c, t


def forward(g, w, t, thr=1e-7, iters=500):
    with Graph(g.row_ptr, g.col, weights=w) as h:
        r = np.empty(g.n, np.float32)
        st = h.weighted_page_rank(t, r, D, thr, iters, record_errors=True)
    return r, st


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_weighted_forward_fixed_sweeps_and_converged(gpu, wgraph):
    g, w, c, t = wgraph
    for tele in (None, t):
        # 12 fixed sweeps from r0 = t, against the FP64 iteration with the same start
        with Graph(g.row_ptr, g.col, weights=w) as h:
            r = np.empty(g.n, np.float32)
            st = h.weighted_page_rank(tele, r, D, 0.0, 12)
        assert st.iterations == 12
        tt = None if tele is None else tele.astype(np.float64)
        ref, _, _ = O.pr_f64(g.row_ptr, g.col, weights=w, teleport=tt, damping=D, tol=0.0, max_iters=12)
        assert np.abs(r - ref).max() < 1e-6 and np.abs(r - ref).sum() < 1e-5
        # converged
        r, st = forward(g, w, tele)
        # 1e-7 is near the FP32 floor of an L1 change over n ranks of ~1/n: converged, or stalled at that floor
        assert st.final_error < 1e-6
        ref, _, _ = O.pr_f64(g.row_ptr, g.col, weights=w, teleport=tt, damping=D, tol=1e-15)
        assert np.abs(r - ref).max() < 1e-6 and np.abs(r - ref).sum() < 1e-5
        # per-sweep FP64 errors are L1 changes of the FP32 iterates
        assert np.all(np.diff(st.errors[:5]) < 0)


@pytest.mark.parametrize("solver", ["gmres", "jacobi"])
def test_vjp_matches_fp64_oracle(gpu, wgraph, solver, monkeypatch):
    """Both adjoint solvers: restarted GMRES (default) and the fixed-point
    iteration (NWGPU_VJP_SOLVER=jacobi)."""
    monkeypatch.setenv("NWGPU_VJP_SOLVER", solver)
    g, w, c, t = wgraph
    r, _ = forward(g, w, t)
    dw = np.empty(g.nnz, np.float32)
    dt = np.empty(g.n, np.float32)
    # the adjoint lives on c's scale (O(1) entries), not a distribution's: a relative threshold
    thr = 1e-6 * float(np.abs(c).sum())
    with Graph(g.row_ptr, g.col, weights=w) as h:
        st = h.page_rank_vjp(r, c, dw, dt, D, thr, 2000, record_errors=True)
    assert st.converged
    r64, _, _ = O.pr_f64(g.row_ptr, g.col, weights=w, teleport=t.astype(np.float64), damping=D, tol=1e-15)
    lam, dt64, dw64 = O.vjp_f64(g.row_ptr, g.col, r64, c.astype(np.float64), weights=w, damping=D, tol=1e-13)
    assert rel_err(dt, dt64) < 1e-4
    assert rel_err(dw, dw64) < 1e-4
    # operator applications: GMRES about as many as the forward's sweeps
    assert st.iterations < (60 if solver == "gmres" else 200)
    assert st.final_error < thr


def loss64(g, w, t, c):
    r, _, _ = O.pr_f64(g.row_ptr, g.col, weights=w, teleport=t, damping=D, tol=1e-15)
    return float(np.dot(c.astype(np.float64), r))


def test_vjp_matches_finite_differences(gpu):
    # 64 random edges and 8 teleport entries, FP64 central differences, h = 1e-3
    g = G.rmat(11, 16, 5)
    w = G.edge_weights(g.nnz, seed=77)
    rng = np.random.default_rng(8)
    c = rng.standard_normal(g.n).astype(np.float32)
    t = np.full(g.n, 1.0 / g.n)
    r, _ = forward(g, w, t.astype(np.float32), thr=1e-9, iters=1000)
    dw = np.empty(g.nnz, np.float32)
    dt = np.empty(g.n, np.float32)
    with Graph(g.row_ptr, g.col, weights=w) as h:
        h.page_rank_vjp(r, c, dw, dt, D, 1e-7 * float(np.abs(c).sum()), 3000)
    h_ = 1e-3
    scale_w = np.abs(dw).max()
    for k in rng.choice(g.nnz, 64, replace=False):
        wp, wm = w.copy(), w.copy()
        wp[k] += h_
        wm[k] -= h_
        # the raw FP32 weights stay exactly representable steps apart: use the actual step
        step = float(wp[k]) - float(wm[k])
        fd = (loss64(g, wp, t, c) - loss64(g, wm, t, c)) / step
        assert abs(dw[k] - fd) <= 1e-4 * max(abs(fd), 1e-2 * scale_w), (k, dw[k], fd)
    for v in rng.choice(g.n, 8, replace=False):
        tp, tm = t.copy(), t.copy()
        tp[v] += h_
        tm[v] -= h_
        fd = (loss64(g, w, tp, c) - loss64(g, w, tm, c)) / (2 * h_)
        assert abs(dt[v] - fd) <= 1e-4 * max(abs(fd), 1e-2 * np.abs(dt).max()), (v, dt[v], fd)


class WeightedPageRank:
    """Test-side torch.autograd.Function: r = weighted PageRank(w, t) on a
    fixed graph structure; backward is nwgpu_pr_vjp (implicit adjoint)."""

    @staticmethod
    def make(torch, row_ptr, col):
        class Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, w, t):
                h = Graph(row_ptr, col, weights=w.detach().cpu().numpy())
                r = torch.empty(len(row_ptr) - 1, dtype=torch.float32, device=w.device)
                h.weighted_page_rank(t.detach(), r, D, 1e-8, 2000)
                ctx.h = h
                ctx.save_for_backward(r)
                return r

            @staticmethod
            def backward(ctx, grad_r):
                (r,) = ctx.saved_tensors
                dw = torch.empty(ctx.h.nnz, dtype=torch.float32, device=r.device)
                dt = torch.empty(ctx.h.n, dtype=torch.float32, device=r.device)
                g = grad_r.contiguous()
                ctx.h.page_rank_vjp(r, g, dw, dt, D, 1e-7 * float(g.abs().sum()), 3000)
                torch.cuda.synchronize()
                ctx.h.release()
                return dw, dt

        return Fn


def test_torch_autograd_function(gpu):
    import torch
    g = G.rmat(12, 16, 3)
    dev = torch.device("cuda")
    w = torch.from_numpy(G.edge_weights(g.nnz, seed=5)).to(dev).requires_grad_(True)
    t = torch.full((g.n,), 1.0 / g.n, device=dev).requires_grad_(True)
    c = torch.from_numpy(np.random.default_rng(1).standard_normal(g.n).astype(np.float32)).to(dev)
    Fn = WeightedPageRank.make(torch, g.row_ptr, g.col)
    loss = (Fn.apply(w, t) * c).sum()
    loss.backward()
    r64, _, _ = O.pr_f64(g.row_ptr, g.col, weights=w.detach().cpu().numpy(), teleport=np.full(g.n, 1.0 / g.n),
                         damping=D, tol=1e-15)
    _, dt64, dw64 = O.vjp_f64(g.row_ptr, g.col, r64, c.cpu().numpy().astype(np.float64),
                              weights=w.detach().cpu().numpy(), damping=D, tol=1e-13)
    assert rel_err(w.grad.cpu().numpy(), dw64) < 1e-4
    assert rel_err(t.grad.cpu().numpy(), dt64) < 1e-4


def test_device_pointers_and_launch_modes(gpu, wgraph):
    import torch
    g, w, c, t = wgraph
    dev = torch.device("cuda")
    r_h, _ = forward(g, w, t)
    with Graph(torch.from_numpy(g.row_ptr.view(np.int32)).to(dev), torch.from_numpy(g.col.view(np.int32)).to(dev),
               weights=torch.from_numpy(w).to(dev)) as h:
        r_d = torch.empty(g.n, dtype=torch.float32, device=dev)
        h.weighted_page_rank(torch.from_numpy(t).to(dev), r_d, D, 1e-7, 500, launch="stream")
        assert np.array_equal(r_d.cpu().numpy(), r_h)
        dw_d = torch.empty(g.nnz, dtype=torch.float32, device=dev)
        h.page_rank_vjp(r_d, torch.from_numpy(c).to(dev), dw_d, None, D, 1e-6 * float(np.abs(c).sum()), 2000)
        dw_h = np.empty(g.nnz, np.float32)
        h.page_rank_vjp(r_h, c, dw_h, None, D, 1e-6 * float(np.abs(c).sum()), 2000, launch="stream")
        assert np.array_equal(dw_d.cpu().numpy(), dw_h)


def test_unsupported_cases(gpu, wgraph):
    g, w, c, t = wgraph
    r = np.empty(g.n, np.float32)
    with Graph(g.row_ptr, g.col) as h:  # no weights
        with pytest.raises(NwgpuError) as ei:
            h.weighted_page_rank(None, r)
        assert ei.value.status == N.ERR_UNSUPPORTED
    with Graph(g.row_ptr, g.col, weights=w, relabel=False) as h:
        with pytest.raises(NwgpuError) as ei:
            h.weighted_page_rank(None, r)
        assert ei.value.status == N.ERR_UNSUPPORTED
    # a directed graph: its out-rows are not in the relabelled (in-degree) order
    rng = np.random.default_rng(0)
    src = rng.integers(0, 5000, 40000).astype(np.uint32)
    dst = (rng.pareto(1.5, 40000) * 50).astype(np.uint32) % 5000
    dg = G.from_edges(src, dst, 5000)
    wd = G.edge_weights(dg.nnz, seed=3)
    with Graph(dg.row_ptr, dg.col, weights=wd) as h:
        rr = np.empty(dg.n, np.float32)
        h.weighted_page_rank(None, rr, D, 1e-7, 300)
        ref, _, _ = O.pr_f64(dg.row_ptr, dg.col, weights=wd, damping=D, tol=1e-15)
        assert np.abs(rr - ref).max() < 1e-6
        with pytest.raises(NwgpuError) as ei:
            h.page_rank_vjp(rr, np.ones(dg.n, np.float32), None, np.empty(dg.n, np.float32))
        assert ei.value.status == N.ERR_UNSUPPORTED
    with pytest.raises(NwgpuError):
        with Graph(g.row_ptr, g.col, weights=w) as h:
            h.page_rank_vjp(r, None, None, None)
