"""Parity of the B200 engine with NWGraph's page_rank, through the C ABI.

Bar: FP32 scores within 1e-6 max-abs and 1e-5 L1 of the
reference after a fixed sweep count, the same top-100 order apart from ties
inside that tolerance, and the same stopping sweep for threshold runs. The
reference is page_rank_v10 (Jacobi; its outputs are the committed fixtures,
and at larger sizes the C restatement pinned to it bit for bit in
test_oracle.py). Summation order inside a row differs from the CPU's serial
order, so equality is within tolerance, not bitwise.
"""
import threading
import time

import numpy as np
import pytest

import oracle as O
from conftest import REFDATA_NAMES
from nwgraph_b200 import Graph, NwgpuError, graphs as G
from nwgraph_b200 import _native as N

pytestmark = pytest.mark.gpu

MAX_ABS = 1e-6
L1 = 1e-5
# Per-sweep L1 errors sum n FP32 rank differences whose last bits depend on the
# order of the row sums, so they agree to ~1e-7 absolute, not bit for bit.
ERR_ATOL = 1e-6
ERR_RTOL = 1e-4


def solve(rp, cl, deg, thr=0.0, iters=20, launch="graph", damping=0.85, relabel=True):
    with Graph(rp, cl, relabel=relabel) as g:
        out = np.empty(len(rp) - 1, np.float32)
        st = g.page_rank(deg, out, damping, thr, iters, launch=launch, record_errors=True)
    return out, st


def assert_close(a, b, max_abs=MAX_ABS, l1=L1):
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))
    assert d.max() <= max_abs, f"max-abs {d.max():.3e}"
    assert d.sum() <= l1, f"L1 {d.sum():.3e}"


def assert_parity_or_more_accurate(gpu, ref, rp, cl, iters, damping=0.85):
    """For hub graphs where the reference's serial FP32 row sums are themselves
    off by more than the tolerance: the engine must be within tolerance of the
    reference or at least as close as the reference to exact arithmetic (FP64
    Jacobi with the same sweep count)."""
    exact, _, _ = O.pr_f64(rp, cl, damping=damping, tol=0.0, max_iters=iters)
    e_ref = np.abs(ref.astype(np.float64) - exact)
    e_gpu = np.abs(gpu.astype(np.float64) - exact)
    d = np.abs(gpu.astype(np.float64) - ref.astype(np.float64))
    if d.max() <= MAX_ABS and d.sum() <= L1:
        return
    assert e_ref.max() > MAX_ABS, "the reference is accurate here, so the engine must match it"
    assert e_gpu.max() <= e_ref.max() * 1.01 + 1e-9, (e_gpu.max(), e_ref.max())
    assert e_gpu.sum() <= e_ref.sum() * 1.01 + 1e-8, (e_gpu.sum(), e_ref.sum())


HUB_GRAPHS = {"star"}


def top_k_consistent(gpu, ref, k=100, tol=MAX_ABS):
    """Top-k order equal except for swaps of values within tol."""
    order_r = np.argsort(-ref.astype(np.float64), kind="stable")[:k]
    order_g = np.argsort(-gpu.astype(np.float64), kind="stable")[:k]
    for a, b in zip(order_r, order_g):
        if a != b:
            assert abs(float(ref[a]) - float(ref[b])) <= tol, (a, b)


def test_karate_golden(gpu, karate):
    r, st = solve(karate["row_ptr"], karate["col"], karate["deg"], thr=1e-7, iters=100)
    assert st.converged
    # the unit test's own bar (test/page_rank_test.cpp:98-101)
    assert np.allclose(r, karate["answer"], rtol=5e-3, atol=0)
    r20, _ = solve(karate["row_ptr"], karate["col"], karate["deg"], iters=20)
    assert_close(r20, karate["v10_20"])


@pytest.mark.parametrize("name", ["rmat8", "rmat10", "grid", "star", "path", "directed", "isolated"])
@pytest.mark.parametrize("launch", ["graph", "stream"])
def test_small_fixtures(gpu, small_graphs, name, launch):
    g = small_graphs[name]
    close = (lambda a, b, k: assert_parity_or_more_accurate(a, b, g["row_ptr"], g["col"], k)) if name in HUB_GRAPHS \
        else (lambda a, b, k: assert_close(a, b))
    r, st = solve(g["row_ptr"], g["col"], g["deg"], iters=20, launch=launch)
    assert st.iterations == 20
    close(r, g["v10_20"], 20)
    top_k_consistent(r, g["v10_20"])
    r, st = solve(g["row_ptr"], g["col"], g["deg"], thr=1e-4, iters=100, launch=launch)
    assert st.iterations == int(g["v10_thr_iters"][0])
    if name not in HUB_GRAPHS:  # a hub's serial FP32 sum shifts the reference's error trace too
        assert np.allclose(st.errors, g["v10_thr_errors"], rtol=ERR_RTOL, atol=ERR_ATOL)
    close(r, g["v10_thr"], st.iterations)


@pytest.mark.parametrize("name", REFDATA_NAMES)
def test_reference_test_matrices(gpu, refdata, name):
    """The Matrix Market matrices of the reference's own test data, loaded as its
    driver loads them, against NWGraph's page_rank_v10 outputs on them."""
    g = refdata[name]
    r, st = solve(g["row_ptr"], g["col"], g["deg"], iters=20)
    assert st.iterations == 20
    assert_close(r, g["v10_20"])
    r, st = solve(g["row_ptr"], g["col"], g["deg"], thr=1e-4, iters=100)
    assert st.iterations == int(g["v10_thr_iters"][0])
    assert np.allclose(st.errors, g["v10_thr_errors"], rtol=ERR_RTOL, atol=ERR_ATOL)
    assert_close(r, g["v10_thr"])


@pytest.mark.parametrize("name", ["rmat10", "directed", "isolated", "grid"])
def test_relabel_off_matches(gpu, small_graphs, name):
    g = small_graphs[name]
    r, st = solve(g["row_ptr"], g["col"], g["deg"], iters=20, relabel=False)
    assert_close(r, g["v10_20"])


@pytest.mark.parametrize("scale", [12, 14, 16])
def test_rmat_vs_oracle(gpu, scale):
    g = G.rmat(scale, 16, 42)
    deg = g.out_degree()
    ref, it, errs = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 20)
    r, st = solve(g.row_ptr, g.col, deg, iters=20)
    assert st.iterations == 20
    assert_close(r, ref)
    top_k_consistent(r, ref)
    assert np.allclose(st.errors, errs, rtol=ERR_RTOL, atol=ERR_ATOL)
    # against the FP64 power iteration (reported, bounded loosely: FP32 at 20 sweeps)
    r64, _, _ = O.pr_f64(g.row_ptr, g.col, tol=1e-14)
    assert np.abs(r - r64).max() < 1e-4


def test_threshold_run_matches_oracle_sweeps(gpu):
    g = G.rmat(15, 16, 9)
    deg = g.out_degree()
    ref, it, errs = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 1e-4, 100)
    r, st = solve(g.row_ptr, g.col, deg, thr=1e-4, iters=100)
    assert st.iterations == it and st.converged
    assert st.final_error < 1e-4 <= errs[-2]
    assert_close(r, ref)


def test_hub_rows_span_many_tiles(gpu):
    """A star whose hub row is ~25 tiles long exercises the cross-tile finaliser."""
    n = 50_001
    s = np.zeros(n - 1, np.uint32)
    d = np.arange(1, n, dtype=np.uint32)
    g = G.from_edges(s, d, n, symmetrize=True)
    deg = g.out_degree()
    ref, _, _ = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 30)
    r, _ = solve(g.row_ptr, g.col, deg, iters=30)
    assert_parity_or_more_accurate(r, ref, g.row_ptr, g.col, 30)
    # a few more hubs plus leaves, rows landing on arbitrary tile offsets
    rng = np.random.default_rng(0)
    hubs = rng.integers(0, 2000, size=6)
    src = np.concatenate([np.full(3000 + 997 * i, h, np.uint32) for i, h in enumerate(hubs)])
    dst = rng.integers(0, 60_000, size=len(src)).astype(np.uint32)
    g = G.from_edges(src, dst, 60_000, symmetrize=True)
    deg = g.out_degree()
    ref, _, _ = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 20)
    for relabel in (True, False):
        r, _ = solve(g.row_ptr, g.col, deg, relabel=relabel)
        assert_parity_or_more_accurate(r, ref, g.row_ptr, g.col, 20)


def test_bitwise_reproducible_and_launch_modes_agree(gpu):
    g = G.rmat(14, 16, 3)
    deg = g.out_degree()
    a, _ = solve(g.row_ptr, g.col, deg, launch="graph")
    b, _ = solve(g.row_ptr, g.col, deg, launch="graph")
    c, _ = solve(g.row_ptr, g.col, deg, launch="stream")
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(a.view(np.uint32), c.view(np.uint32))


def test_resident_graph_reused_and_damping_changes(gpu):
    g = G.rmat(12, 16, 5)
    deg = g.out_degree()
    with Graph(g.row_ptr, g.col) as h:
        for d in (0.85, 0.5, 0.85, 0.99):
            out = np.empty(g.n, np.float32)
            h.page_rank(deg, out, d, 0.0, 15)
            ref, _, _ = O.jacobi_f32(g.row_ptr, g.col, deg, d, 0.0, 15)
            assert_close(out, ref)


def test_device_pointers(gpu):
    import torch
    g = G.rmat(13, 16, 11)
    deg = g.out_degree()
    ref, _, _ = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 20)
    dev = torch.device("cuda")
    rp = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    cl = torch.from_numpy(g.col.view(np.int32)).to(dev)
    dg = torch.from_numpy(deg.view(np.int32)).to(dev)
    out = torch.empty(g.n, dtype=torch.float32, device=dev)
    with Graph(rp, cl) as h:
        h.page_rank(dg, out, 0.85, 0.0, 20)
    torch.cuda.synchronize()
    assert_close(out.cpu().numpy(), ref)


def test_edge_cases(gpu):
    # one vertex, no edges: rank = base after every sweep
    r, st = solve(np.array([0, 0], np.uint32), np.zeros(0, np.uint32), np.zeros(1, np.uint32), iters=5)
    assert st.iterations == 5 and abs(float(r[0]) - np.float32(0.15)) < 1e-7
    # all isolated
    n = 5000
    r, st = solve(np.zeros(n + 1, np.uint32), np.zeros(0, np.uint32), np.zeros(n, np.uint32), thr=1e-4, iters=50)
    ref, it, _ = O.jacobi_f32(np.zeros(n + 1, np.uint32), np.zeros(0, np.uint32), np.zeros(n, np.uint32), 0.85,
                              1e-4, 50)
    assert st.iterations == it
    assert_close(r, ref)
    # max_iters = 0: ranks are the initial 1/n and no sweep runs
    g = G.rmat(8, 16, 1)
    r, st = solve(g.row_ptr, g.col, g.out_degree(), iters=0)
    assert st.iterations == 0 and np.all(r == np.float32(1.0 / g.n))
    # a huge threshold stops after the first sweep
    r, st = solve(g.row_ptr, g.col, g.out_degree(), thr=1e9, iters=50)
    assert st.iterations == 1 and st.converged


def test_invalid_graphs_rejected(gpu):
    with pytest.raises(NwgpuError) as ei:
        Graph(np.array([0, 2, 3], np.uint32), np.array([1, 7, 0], np.uint32))
    assert ei.value.status == N.ERR_INVALID_GRAPH and "col" in str(ei.value)
    with pytest.raises(NwgpuError) as ei:
        Graph(np.array([0, 2, 1, 3], np.uint32), np.array([1, 0, 2], np.uint32))
    assert ei.value.status == N.ERR_INVALID_GRAPH
    with pytest.raises(NwgpuError) as ei:
        Graph(np.array([0, 1, 2], np.uint32), np.array([1, 0, 0], np.uint32), nnz=3)
    assert ei.value.status == N.ERR_INVALID_GRAPH


def test_bad_arguments(gpu):
    g = G.rmat(6, 4, 1)
    with Graph(g.row_ptr, g.col) as h:
        with pytest.raises(ValueError):
            h.page_rank(g.out_degree()[:-1], np.empty(g.n, np.float32))
        with pytest.raises(NwgpuError) as ei:
            h.page_rank(g.out_degree(), np.empty(g.n, np.float32), damping_factor=1.5)
        assert ei.value.status == N.ERR_INVALID_ARG


def test_abort_from_another_thread(gpu):
    g = G.rmat(14, 16, 2)
    deg = g.out_degree()
    out = np.empty(g.n, np.float32)
    with Graph(g.row_ptr, g.col) as h:
        t = threading.Timer(0.3, h.abort)
        t.start()
        t0 = time.time()
        with pytest.raises(NwgpuError) as ei:
            h.page_rank(deg, out, 0.85, 0.0, 2_000_000)
        t.join()
        assert ei.value.status == N.ERR_ABORTED
        assert time.time() - t0 < 30
        # the handle stays usable after an abort
        h.page_rank(deg, out, 0.85, 0.0, 3)


@pytest.mark.slow
def test_scale20_properties(gpu):
    g = G.rmat(20, 16, 42)
    deg = g.out_degree()
    ref, _, errs = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 20)
    r, st = solve(g.row_ptr, g.col, deg)
    assert_close(r, ref)
    top_k_consistent(r, ref)
    assert np.allclose(st.errors, errs, rtol=ERR_RTOL, atol=ERR_ATOL)
    # leak semantics: mass is lost only through isolated/dangling vertices
    assert abs(float(r.astype(np.float64).sum()) - float(ref.astype(np.float64).sum())) < 1e-5


@pytest.mark.parametrize("sweep", ["blocked", "binned", "binned_hot", "base", "hot", "hot512"])
def test_sweep_variants_agree(gpu, sweep, monkeypatch):
    """Every sweep kernel variant (degree-binned, merge-path with L1 hot ids,
    merge-path with the hot ids in shared memory) meets the same bar."""
    monkeypatch.setenv("NWGPU_SWEEP", sweep)
    g = G.rmat(15, 16, 77)
    deg = g.out_degree()
    ref, it, errs = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 20)
    r, st = solve(g.row_ptr, g.col, deg)
    assert_close(r, ref)
    assert np.allclose(st.errors, errs, rtol=ERR_RTOL, atol=ERR_ATOL)
    a, _ = solve(g.row_ptr, g.col, deg)
    assert np.array_equal(a.view(np.uint32), r.view(np.uint32))
    # a hub spanning many tiles / chunks
    n = 40_001
    s = np.zeros(n - 1, np.uint32)
    hub = G.from_edges(s, np.arange(1, n, dtype=np.uint32), n, symmetrize=True)
    ref, _, _ = O.jacobi_f32(hub.row_ptr, hub.col, hub.out_degree(), 0.85, 0.0, 10)
    r, _ = solve(hub.row_ptr, hub.col, hub.out_degree(), iters=10)
    assert_parity_or_more_accurate(r, ref, hub.row_ptr, hub.col, 10)


@pytest.mark.parametrize("hot_ids", ["-1", "0", "4", "1000", "40000"])
def test_binned_hot_staging_is_exact(gpu, hot_ids, monkeypatch):
    """Staging the hub contributions in shared memory changes where each value
    is read from, not which values are summed or in what order: the ranks equal
    the plain binned sweep's bit for bit, whatever the staged id count."""
    g = G.rmat(16, 16, 5)
    deg = g.out_degree()
    monkeypatch.setenv("NWGPU_SWEEP", "binned")
    a, _ = solve(g.row_ptr, g.col, deg)
    monkeypatch.setenv("NWGPU_SWEEP", "binned_hot")
    if hot_ids != "-1":
        monkeypatch.setenv("NWGPU_HOT_IDS", hot_ids)
    b, _ = solve(g.row_ptr, g.col, deg)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("graph", ["rmat16", "hubs"])
def test_binned_launch_shapes_and_modes_agree(gpu, graph, monkeypatch):
    """The binned sweep with 256-thread CTAs (hubs through L1) and with one
    1024-thread CTA per SM (hubs staged in shared memory), in CUDA-graph and
    stream mode, sum the same values in the same order: bitwise equal ranks.
    The hub graph splits long rows into many chunks (rows of more than 32
    chunks are finished by a warp, the others by a thread)."""
    if graph == "rmat16":
        g = G.rmat(16, 16, 9)
    else:  # long rows split into many chunks, plus every bin populated
        rng = np.random.default_rng(3)
        src = np.concatenate([np.full(5000 + 1500 * i, i, np.uint32) for i in range(5)] +
                             [np.full(40_000, 7, np.uint32)] +
                             [rng.integers(0, 70_000, 200_000).astype(np.uint32)])
        dst = rng.integers(0, 70_000, len(src)).astype(np.uint32)
        g = G.from_edges(src, dst, 70_000, symmetrize=True)
    deg = g.out_degree()
    monkeypatch.setenv("NWGPU_SWEEP", "binned")
    a, sa = solve(g.row_ptr, g.col, deg)
    monkeypatch.setenv("NWGPU_SWEEP", "binned_hot")
    b, sb = solve(g.row_ptr, g.col, deg)
    c, sc = solve(g.row_ptr, g.col, deg, launch="stream")
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(b.view(np.uint32), c.view(np.uint32))
    # FP64 residuals: the same terms, grouped by CTA differently
    assert np.allclose(sa.errors, sb.errors, rtol=1e-12, atol=0)
    ref, _, errs = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 20)
    assert_parity_or_more_accurate(b, ref, g.row_ptr, g.col, 20)
    # repeated solves on fresh handles
    for _ in range(2):
        d, _ = solve(g.row_ptr, g.col, deg)
        assert np.array_equal(d.view(np.uint32), b.view(np.uint32))


def boundary_graph(seed=17):
    """A directed graph whose row lengths sit on and beside every bin and window boundary of the binned sweep
    (4-entry lanes, the G-bins' 2G/4G edges, bin 0's 128/129, 256-entry windows, the long-row cut-off 2048 and
    1024-entry chunks), several rows of each, so that after relabelling the rows start at every offset mod 4."""
    rng = np.random.default_rng(seed)
    lengths = [1, 2, 3, 4, 5, 7, 8, 9, 15, 16, 17, 31, 32, 33, 63, 64, 65, 127, 128, 129, 130, 131, 255, 256, 257,
               511, 512, 513, 1023, 1024, 1025, 2047, 2048, 2049, 2050, 3071, 3072, 3073, 4096, 4097, 9000]
    lens = np.array([L for L in lengths for _ in range(5)] + [0] * 40, np.int64)
    rng.shuffle(lens)
    n = 6000
    lens = np.concatenate([lens, rng.integers(0, 12, n - len(lens))])
    rp = np.zeros(n + 1, np.uint32)
    rp[1:] = np.cumsum(lens)
    cl = rng.integers(0, n - 50, int(rp[-1])).astype(np.uint32)  # the last 50 vertices have no out-edges
    deg = np.bincount(cl, minlength=n).astype(np.uint32)
    return rp, cl, deg


@pytest.mark.parametrize("env", [{}, {"NWGPU_BIN0_ROWS": "1"}, {"NWGPU_LONG_ROW": "256", "NWGPU_CHUNK_ENTRIES": "256"},
                                 {"NWGPU_SWEEP": "binned"}])
def test_rows_at_bin_and_window_boundaries(gpu, monkeypatch, env):
    """Rows of every boundary length at every start alignment: the 128-bit id windows (long-row chunks, bin 0),
    the G-bins and the empty rows against page_rank_v10 restated, at a fixed sweep count and at threshold 1e-5
    with the same stopping sweep; the graph launch and the stream launch give the same bits; the weighted mode's
    SpMV against FP64 row sums."""
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    rp, cl, deg = boundary_graph()
    a, _ = solve(rp, cl, deg, 0.0, 20)
    b, _ = solve(rp, cl, deg, 0.0, 20, launch="stream")
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    ref, _, _ = O.jacobi_f32(rp, cl, deg, 0.85, 0.0, 20)
    assert_close(a, ref)
    r, st = solve(rp, cl, deg, 1e-5, 200)
    ref, it, _ = O.jacobi_f32(rp, cl, deg, 0.85, 1e-5, 200)
    assert st.iterations == it
    assert_close(r, ref)
    # the weighted mode of the same walk: SpMV against FP64 row sums
    w = G.edge_weights(len(cl), seed=3)
    x = np.random.default_rng(5).standard_normal(len(rp) - 1).astype(np.float32)
    with Graph(rp, cl, weights=w) as h:
        y = np.empty(len(rp) - 1, np.float32)
        h.spmv(x, y)
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp.astype(np.int64)))
    t = w.astype(np.float64) * x.astype(np.float64)[cl]
    exact = np.bincount(rows, weights=t, minlength=len(rp) - 1)
    mag = np.bincount(rows, weights=np.abs(t), minlength=len(rp) - 1)
    assert np.all(np.abs(y - exact) <= 1e-6 * mag + 1e-30)
