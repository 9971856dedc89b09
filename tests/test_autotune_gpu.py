"""Autotuner (NWGPU_GRAPH_AUTOTUNE) of the binned sweep (long-row cut-offs,
bin-0 rows per warp, launch shape, hub tiers) and, with NWGPU_SWEEP=blocked, of
the blocked sweep (entries in flight, piece size). Launch shape, hub tiers and
the blocked knobs do not change the summation order; the long-row cut-offs
and bin-0 rows per warp do, so a tuned graph must give, bit for bit, the ranks
of an untuned graph created with the tuner's choice (NWGPU_LONG_ROW,
NWGPU_CHUNK_ENTRIES, NWGPU_BIN0_ROWS), and every choice must keep parity with
page_rank_v10 restated. Choices are cached per graph
signature in the process and, with NWGPU_TUNE_CACHE, in a file that a later
process reuses."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
from nwgraph_b200 import Graph, graphs as G

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def solve(g, deg, **kw):
    with Graph(g.row_ptr, g.col, **kw) as h:
        out = np.empty(g.n, np.float32)
        h.page_rank(deg, out, 0.85, 0.0, 20)
        return out, h.info()


KEYS = ("sweep_threads", "hub_smem_ids", "hub_l1_ids", "long_row_entries", "chunk_entries", "bin0_rows_per_warp",
        "block_loads", "block_piece_entries")


def test_tuned_ranks_are_bitwise_equal_and_cached(gpu, monkeypatch):
    monkeypatch.delenv("NWGPU_TUNE_CACHE", raising=False)
    g = G.rmat(17, 16, 5)
    deg = g.out_degree()
    r0, i0 = solve(g, deg)
    r1, i1 = solve(g, deg, autotune=True)
    r2, i2 = solve(g, deg, autotune=True)
    assert i0["tuned"] == 0 and i0["binned"] == 1
    assert (i0["long_row_entries"], i0["chunk_entries"], i0["bin0_rows_per_warp"]) == (2048, 1024, 2)
    assert i1["tuned"] in (1, 2) and i1["tuned_us_per_sweep"] > 0
    assert i2["tuned"] == 2  # same signature: taken from the cache
    for k in KEYS:
        assert i1[k] == i2[k]
    assert np.array_equal(r1.view(np.uint32), r2.view(np.uint32))
    # an untuned graph with the tuner's cut-offs sums in the same order
    monkeypatch.setenv("NWGPU_LONG_ROW", str(i1["long_row_entries"]))
    monkeypatch.setenv("NWGPU_CHUNK_ENTRIES", str(i1["chunk_entries"]))
    monkeypatch.setenv("NWGPU_BIN0_ROWS", str(i1["bin0_rows_per_warp"]))
    r3, i3 = solve(g, deg)
    assert i3["tuned"] == 0
    assert np.array_equal(r1.view(np.uint32), r3.view(np.uint32))
    ref, _, _ = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 20)
    for r in (r0, r1):
        assert np.abs(r.astype(np.float64) - ref).max() <= 1e-6


@pytest.mark.parametrize("long_row,chunk", [(256, 256), (1024, 512), (4096, 2048), (8192, 2048)])
def test_long_row_cutoffs_keep_parity(gpu, monkeypatch, long_row, chunk):
    """Rows of more than long_row entries are cut into chunks of `chunk` entries; at RMAT scale 17 the cut-offs
    move rows of 257 to 8192 entries between the warp-per-row bin and the chunks (rows of more than 32 chunks
    get a warp in the finishing kernel at 256-entry chunks)."""
    monkeypatch.setenv("NWGPU_LONG_ROW", str(long_row))
    monkeypatch.setenv("NWGPU_CHUNK_ENTRIES", str(chunk))
    g = G.rmat(17, 16, 5)
    deg = g.out_degree()
    with Graph(g.row_ptr, g.col) as h:
        out = np.empty(g.n, np.float32)
        h.page_rank(deg, out, 0.85, 0.0, 20)
        info = h.info()
        assert (info["long_row_entries"], info["chunk_entries"]) == (long_row, chunk)
        ref, _, _ = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 20)
        d = np.abs(out.astype(np.float64) - ref)
        assert d.max() <= 1e-6 and d.sum() <= 1e-5
        st = h.page_rank(deg, out, 0.85, 1e-4, 100)
        ref, it, _ = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 1e-4, 100)
        assert st.iterations == it
        d = np.abs(out.astype(np.float64) - ref)
        assert d.max() <= 1e-6 and d.sum() <= 1e-5


@pytest.mark.parametrize("long_row,chunk", [(2048, 1024), (8192, 2048)])
def test_bin0_warp_per_row_keeps_parity(gpu, monkeypatch, long_row, chunk):
    """NWGPU_BIN0_ROWS=1: rows of 129 entries to the long-row cut-off get a whole warp each (256-entry windows,
    a 32-lane tree) instead of half a warp; plain PageRank against page_rank_v10 restated at a fixed sweep count
    and at threshold 1e-4 with equal sweep counts, and the weighted sweep's SpMV against FP64 row sums."""
    monkeypatch.setenv("NWGPU_BIN0_ROWS", "1")
    monkeypatch.setenv("NWGPU_LONG_ROW", str(long_row))
    monkeypatch.setenv("NWGPU_CHUNK_ENTRIES", str(chunk))
    g = G.rmat(17, 16, 5)
    deg = g.out_degree()
    with Graph(g.row_ptr, g.col) as h:
        out = np.empty(g.n, np.float32)
        h.page_rank(deg, out, 0.85, 0.0, 20)
        info = h.info()
        assert (info["bin0_rows_per_warp"], info["long_row_entries"]) == (1, long_row)
        ref, _, _ = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 20)
        d = np.abs(out.astype(np.float64) - ref)
        assert d.max() <= 1e-6 and d.sum() <= 1e-5
        again = np.empty(g.n, np.float32)
        h.page_rank(deg, again, 0.85, 0.0, 20, launch="stream")
        assert np.array_equal(out.view(np.uint32), again.view(np.uint32))
        st = h.page_rank(deg, out, 0.85, 1e-4, 100)
        ref, it, _ = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 1e-4, 100)
        assert st.iterations == it
        d = np.abs(out.astype(np.float64) - ref)
        assert d.max() <= 1e-6 and d.sum() <= 1e-5
    w = G.edge_weights(g.nnz, seed=9)
    x = np.random.default_rng(4).standard_normal(g.n).astype(np.float32)
    with Graph(g.row_ptr, g.col, weights=w) as h:
        y = np.empty(g.n, np.float32)
        h.spmv(x, y)
    rows = np.repeat(np.arange(g.n), np.diff(g.row_ptr.astype(np.int64)))
    t = w.astype(np.float64) * x.astype(np.float64)[g.col]
    exact = np.bincount(rows, weights=t, minlength=g.n)
    mag = np.bincount(rows, weights=np.abs(t), minlength=g.n)
    assert np.all(np.abs(y - exact) <= 1e-6 * mag + 1e-30)


def test_bad_bin0_rows_refused(gpu, monkeypatch):
    monkeypatch.setenv("NWGPU_BIN0_ROWS", "3")
    g = G.rmat(12, 16, 5)
    with pytest.raises(Exception, match="bin-0 rows per warp"):
        Graph(g.row_ptr, g.col)


@pytest.mark.parametrize("long_row,chunk", [(255, 1024), (2048, 100), (2048, 1000)])
def test_bad_cutoffs_are_refused(gpu, monkeypatch, long_row, chunk):
    monkeypatch.setenv("NWGPU_LONG_ROW", str(long_row))
    monkeypatch.setenv("NWGPU_CHUNK_ENTRIES", str(chunk))
    g = G.rmat(12, 16, 5)
    with pytest.raises(Exception, match="long-row cut-off"):
        Graph(g.row_ptr, g.col)


def test_environment_settings_take_precedence(gpu, monkeypatch):
    monkeypatch.setenv("NWGPU_SWEEP", "binned")
    g = G.rmat(12, 16, 9)
    _, info = solve(g, g.out_degree(), autotune=True)
    assert info["tuned"] == 0 and info["sweep_threads"] == 256


CHILD = r"""
import json, sys
sys.path.insert(0, {root!r})
import numpy as np
from nwgraph_b200 import Graph, graphs as G
g = G.grid(90000)
with Graph(g.row_ptr, g.col, autotune=True) as h:
    out = np.empty(g.n, np.float32)
    h.page_rank(g.out_degree(), out, 0.85, 0.0, 5)
    print(json.dumps(h.info()))
"""


def test_cache_file_is_reused_by_another_process(gpu, tmp_path):
    path = tmp_path / "tune.txt"
    env = dict(os.environ, NWGPU_TUNE_CACHE=str(path))
    env.pop("NWGPU_SWEEP", None)
    code = CHILD.format(root=ROOT)
    a = json.loads(subprocess.run([sys.executable, "-c", code], env=env, check=True, capture_output=True,
                                  text=True).stdout.strip().splitlines()[-1])
    assert a["tuned"] == 1 and path.exists()
    lines = path.read_text().strip().splitlines()
    assert len(lines) == 1 and lines[0].startswith("binned sms=")
    b = json.loads(subprocess.run([sys.executable, "-c", code], env=env, check=True, capture_output=True,
                                  text=True).stdout.strip().splitlines()[-1])
    assert b["tuned"] == 2
    for k in KEYS:
        assert a[k] == b[k]



def test_blocked_tuning_bitwise_equal_and_cached(gpu, monkeypatch):
    monkeypatch.delenv("NWGPU_TUNE_CACHE", raising=False)
    monkeypatch.setenv("NWGPU_SWEEP", "blocked")
    g = G.rmat(17, 16, 6)
    deg = g.out_degree()
    r0, i0 = solve(g, deg)
    r1, i1 = solve(g, deg, autotune=True)
    r2, i2 = solve(g, deg, autotune=True)
    assert i0["blocked"] == 1 and i0["tuned"] == 0
    assert i1["tuned"] in (1, 2) and i2["tuned"] == 2
    assert (i1["block_loads"], i1["block_piece_entries"]) == (i2["block_loads"], i2["block_piece_entries"])
    assert np.array_equal(r0.view(np.uint32), r1.view(np.uint32))
    assert np.array_equal(r0.view(np.uint32), r2.view(np.uint32))


@pytest.mark.parametrize("scale", [10, 12, 14])
def test_small_tuned_graphs_stop_where_untuned_ones_do(gpu, monkeypatch, scale):
    """A small graph has few merge-path tiles, so its merge-path sweep writes fewer residual partials than the
    binned sweep's 256-thread shape (four CTAs per SM), which the tuner times and may keep; the handle's partials
    are sized for the larger of its sweeps. The tuned solve must stop at the sweep of an untuned solve with the
    tuner's cut-offs and bin-0 rows per warp, with the same ranks and stopping error, and keep parity with the restated page_rank_v10."""
    monkeypatch.delenv("NWGPU_TUNE_CACHE", raising=False)
    g = G.rmat(scale, 16, 21)
    deg = g.out_degree()

    def run(tune):
        with Graph(g.row_ptr, g.col, autotune=tune) as h:
            out = np.empty(g.n, np.float32)
            st = h.page_rank(deg, out, 0.85, 1e-6, 200)
            return out, st, h.info()

    r1, s1, i1 = run(True)
    assert i1["tuned"] in (1, 2)
    monkeypatch.setenv("NWGPU_LONG_ROW", str(i1["long_row_entries"]))
    monkeypatch.setenv("NWGPU_CHUNK_ENTRIES", str(i1["chunk_entries"]))
    monkeypatch.setenv("NWGPU_BIN0_ROWS", str(i1["bin0_rows_per_warp"]))
    r0, s0, _ = run(False)
    assert s0.converged and s1.converged and s0.iterations == s1.iterations
    assert s0.final_error == s1.final_error
    assert np.array_equal(r0.view(np.uint32), r1.view(np.uint32))
    ref, it, _ = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 1e-6, 200)
    assert s1.iterations == it
    assert np.abs(r1.astype(np.float64) - ref).max() <= 1e-6
