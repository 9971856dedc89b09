"""The oracle, pinned before it is trusted (CPU only).

* page_rank_v1<double> restated vs the karate golden vector of
  test/page_rank_test.cpp:72-75 (same 0.5% relative tolerance as :98-101);
* the FP32 Jacobi restatement vs NWGraph's page_rank_v10 outputs (committed
  fixtures made by tests/golden/make_golden.py from the reference headers),
  bit for bit; the Gauss-Seidel restatement vs page_rank v11 on one thread,
  bit for bit; sweep counts and per-sweep errors of the threshold run;
* when oracle/_ref is present, the same comparisons live on fresh RMAT graphs;
* the FP64 extensions (personalized teleport, weights, implicit adjoint)
  against central finite differences.
"""
import numpy as np
import pytest

import oracle as O
from conftest import REFDATA_NAMES
from nwgraph_b200 import graphs as G


def test_karate_golden_v1(karate):
    r, it = O.v1_f64(karate["row_ptr"], karate["col"], karate["deg"], 0.85, 1e-7, 100)
    assert np.allclose(r, karate["answer"], rtol=5e-3, atol=0)
    # the restatement reproduces the reference's own v1 run bit for bit
    assert np.array_equal(r, karate["v1_f64"])


def test_karate_csr_is_symmetric_156(karate):
    assert int(karate["row_ptr"][-1]) == 156 and len(karate["row_ptr"]) == 35
    assert np.array_equal(karate["deg"], np.diff(karate["row_ptr"]))


@pytest.mark.parametrize("name", ["rmat8", "rmat10", "grid", "star", "path", "directed", "isolated"])
def test_restatement_bitwise_vs_reference_fixtures(small_graphs, name):
    g = small_graphs[name]
    rp, cl, deg = g["row_ptr"], g["col"], g["deg"]
    assert np.array_equal(deg, O.out_degree(rp, cl, len(rp) - 1))
    r, it, _ = O.jacobi_f32(rp, cl, deg, 0.85, 0.0, 20)
    assert it == 20
    assert np.array_equal(r.view(np.uint32), g["v10_20"].view(np.uint32))
    r, it, _ = O.gauss_seidel_f32(rp, cl, deg, 0.85, 0.0, 20)
    assert np.array_equal(r.view(np.uint32), g["v11_20_t1"].view(np.uint32))
    r, it, errs = O.jacobi_f32(rp, cl, deg, 0.85, 1e-4, 100)
    assert it == int(g["v10_thr_iters"][0])
    assert np.array_equal(r.view(np.uint32), g["v10_thr"].view(np.uint32))
    assert np.allclose(errs, g["v10_thr_errors"], rtol=0, atol=6e-11)  # trace prints 10 decimals


@pytest.mark.parametrize("name", REFDATA_NAMES)
def test_restatement_bitwise_on_the_reference_test_matrices(refdata, name):
    """The same pins on the Matrix Market matrices of the reference's own test
    data, loaded as its driver loads them (read_mm<directed>, adjacency<1>)."""
    test_restatement_bitwise_vs_reference_fixtures({name: refdata[name]}, name)


def test_karate_fp32_fixtures(karate):
    r, _, _ = O.jacobi_f32(karate["row_ptr"], karate["col"], karate["deg"], 0.85, 0.0, 20)
    assert np.array_equal(r, karate["v10_20"])
    r, _, _ = O.gauss_seidel_f32(karate["row_ptr"], karate["col"], karate["deg"], 0.85, 0.0, 20)
    assert np.array_equal(r, karate["v11_20_t1"])


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
@pytest.mark.parametrize("scale", [12, 14])
def test_restatement_vs_live_reference(scale):
    g = G.rmat(scale, 16, 42)
    deg = O.ref_build_degrees(g.row_ptr, g.col, 4)
    assert np.array_equal(deg, g.out_degree())
    for nt in (1, 4):
        rr, itr, er, _ = O.ref_page_rank(10, g.row_ptr, g.col, deg, 0.85, 0.0, 20, nt)
        ro, ito, eo = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 20)
        assert itr == ito == 20
        assert np.array_equal(rr.view(np.uint32), ro.view(np.uint32))


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
def test_generator_csr_matches_reference_fill():
    """The generator's rows equal the reference's fill of the same edge list
    (fill_directed sorts rows unstably, so compare rows as sorted sets)."""
    g = G.rmat(10, 16, 42)
    src = np.repeat(np.arange(g.n, dtype=np.uint32), np.diff(g.row_ptr))  # row = destination
    rp, cl = O.ref_fill_adj1(g.col, src, g.n)  # edge col -> row
    assert np.array_equal(rp, g.row_ptr)
    for i in range(0, g.n, 7):
        a, b = rp[i], rp[i + 1]
        assert np.array_equal(np.sort(cl[a:b]), g.col[a:b])


def test_fp64_oracle_is_fixed_point():
    g = G.rmat(9, 16, 1)
    r, it, fe = O.pr_f64(g.row_ptr, g.col, tol=1e-15)
    assert fe < 1e-14
    deg = g.out_degree().astype(np.float64)
    c = np.where(deg > 0, r / np.maximum(deg, 1), 0.0)
    rows = np.repeat(np.arange(g.n), np.diff(g.row_ptr))
    z = np.bincount(rows, weights=c[g.col], minlength=g.n)
    assert np.allclose(0.15 / g.n + 0.85 * z, r, rtol=0, atol=1e-15)


def _weighted_small(seed=0):
    g = G.rmat(7, 8, seed)
    w = G.edge_weights(g.nnz, seed=seed + 1)
    return g, w


def test_vjp_fp64_matches_finite_differences_weights():
    g, w = _weighted_small()
    n = g.n
    rng = np.random.default_rng(2)
    cvec = rng.standard_normal(n)
    t = np.zeros(n)
    t[rng.integers(0, n)] = 1.0
    r, _, _ = O.pr_f64(g.row_ptr, g.col, weights=w, teleport=t, tol=1e-15)
    lam, dt, dw = O.vjp_f64(g.row_ptr, g.col, r, cvec, weights=w, tol=1e-15)
    h = 1e-3
    for k in rng.integers(0, g.nnz, size=12):
        wp = w.astype(np.float64).copy()
        wm = wp.copy()
        wp[k] += h
        wm[k] -= h
        rp_, _, _ = O.pr_f64(g.row_ptr, g.col, weights=wp.astype(np.float32), teleport=t, tol=1e-15)
        rm_, _, _ = O.pr_f64(g.row_ptr, g.col, weights=wm.astype(np.float32), teleport=t, tol=1e-15)
        # the float32 cast of w +- h is not exact; use the realised step
        hp = float(np.float32(wp[k])) - float(w[k])
        hm = float(w[k]) - float(np.float32(wm[k]))
        fd = (cvec @ rp_ - cvec @ rm_) / (hp + hm)
        assert abs(fd - dw[k]) <= 1e-4 * max(abs(dw).max(), 1e-12)


def test_vjp_fp64_matches_finite_differences_teleport():
    g, w = _weighted_small(3)
    n = g.n
    rng = np.random.default_rng(4)
    cvec = rng.standard_normal(n)
    t = rng.uniform(0.5, 1.5, n)
    t /= t.sum()
    r, _, _ = O.pr_f64(g.row_ptr, g.col, weights=w, teleport=t, tol=1e-15)
    lam, dt, _ = O.vjp_f64(g.row_ptr, g.col, r, cvec, weights=w, tol=1e-15, want_dw=False)
    h = 1e-6
    for v in rng.integers(0, n, size=8):
        tp = t.copy()
        tm = t.copy()
        tp[v] += h
        tm[v] -= h
        rp_, _, _ = O.pr_f64(g.row_ptr, g.col, weights=w, teleport=tp, tol=1e-15)
        rm_, _, _ = O.pr_f64(g.row_ptr, g.col, weights=w, teleport=tm, tol=1e-15)
        fd = (cvec @ rp_ - cvec @ rm_) / (2 * h)
        assert abs(fd - dt[v]) <= 1e-6 * max(abs(dt).max(), 1e-12)


def test_build_csr_restatement_matches_reference_golden(csr_golden):
    """oracle.build_csr (edge clean-up + fill restated) against the CSRs the
    reference's own remove_self_loops / uniq / fill built (csr_build.npz)."""
    for name, g in csr_golden.items():
        for f in range(0, 0x20, 2):
            rp, cl, deg = O.build_csr(g["src"], g["dst"], g["n"], f)
            assert np.array_equal(rp, g[f]["row_ptr"]), (name, f)
            assert np.array_equal(cl, g[f]["col"]), (name, f)
            assert np.array_equal(deg, g[f]["deg"]), (name, f)


def test_residual_restatement_matches_reference_v13():
    """oracle.residual_f32 restates page_rank_v13 (experimental/algorithms/
    page_rank.hpp:552-625): bit for bit against the compiled reference on one
    thread, with its iteration count."""
    if not O.ref_available():
        pytest.skip("the reference build (oracle/_ref) is not present")
    for g in (G.rmat(10, 16, 3), G.grid(1000)):
        deg = g.out_degree()
        for thr, iters in ((1e-4, 100), (0.0, 12), (1e-3, 5)):
            r, it, _ = O.residual_f32(g.row_ptr, g.col, deg, 0.85, thr, iters)
            rr, rit, _, _ = O.ref_page_rank(13, g.row_ptr, g.col, deg, 0.85, thr, iters, 1)
            assert it == rit and np.array_equal(r.view(np.uint32), rr.view(np.uint32)), (g.n, thr)


@pytest.mark.skipif(not O.ref_available(fast=True), reason="oracle/_ref not built")
def test_reference_library_input_builder_matches():
    """The benchmark's reference arm builds its RMAT input with the builder copy in the reference library: the
    same CSR as the engine's builder."""
    from nwgraph_b200 import graphs as G
    rp, cl = O.ref_rmat(12, 16, 42)
    g = G.rmat(12, 16, 42)
    assert np.array_equal(rp, g.row_ptr) and np.array_equal(cl, g.col)
