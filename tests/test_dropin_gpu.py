"""The C++20 drop-in layer (include/nwgraph_gpu/page_rank.hpp) on the GPU.

* tests/cpp/dropin_test: a graph type with NWGraph's public CSR members, the
  reference's exact call with the namespace switched to nw::graph::gpu;
* oracle/_ref/dropin_ref: the same call on NWGraph's own adjacency<1> read
  from MatrixMarket with read_mm, next to the reference's page_rank_v10 in the
  same process (built where the reference tree exists; shipped as a binary).
"""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT
from nwgraph_b200 import graphs as G

pytestmark = pytest.mark.gpu

DROPIN = os.path.join(ROOT, "tests", "cpp", "dropin_test")
DROPIN_REF = os.path.join(ROOT, "oracle", "_ref", "dropin_ref")


def write_mtx(path, g):
    rows = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(g.row_ptr))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern general\n")
        f.write(f"{g.n} {g.n} {g.nnz}\n")
        # adjacency<1> groups by the second index: line "j+1 i+1" puts j in row i
        np.savetxt(f, np.stack([g.col.astype(np.int64) + 1, rows + 1], axis=1), fmt="%d")


def test_cpp_dropin_standin_graph(gpu, tmp_path):
    assert os.path.exists(DROPIN), "build() must produce tests/cpp/dropin_test"
    g = G.rmat(13, 16, 21)
    deg = g.out_degree()
    g.row_ptr.tofile(tmp_path / "row_ptr.u32")
    g.col.tofile(tmp_path / "col.u32")
    deg.tofile(tmp_path / "deg.u32")
    res = subprocess.run([DROPIN, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    ranks = np.fromfile(tmp_path / "ranks.f32", np.float32)
    ref, _, _ = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 20)
    d = np.abs(ranks.astype(np.float64) - ref)
    assert d.max() <= 1e-6 and d.sum() <= 1e-5
    # gpu::page_rank_v13: the residual push, within a few thresholds of the reference's v13 (restated)
    v13 = np.fromfile(tmp_path / "ranks_v13.f32", np.float32)
    r13, _, _ = O.residual_f32(g.row_ptr, g.col, deg, 0.85, 1e-4, 100)
    assert np.all(np.abs(v13.astype(np.float64) - r13) <= 4e-4 + 1e-5 * np.abs(r13))


@pytest.mark.skipif(not os.path.exists(DROPIN_REF), reason="oracle/_ref/dropin_ref not built")
@pytest.mark.parametrize("scale", [10, 16])
def test_cpp_dropin_on_reference_adjacency(gpu, tmp_path, scale):
    """Config 1's path: RMAT written as .mtx, read by read_mm into adjacency<1>; the drop-in against
    page_rank_v10 at 20 sweeps, and against page_rank (v11) converged, on top-100 order and on the
    threshold-1e-4 sweep counts (oracle/dropin_ref.cpp, mode o2)."""
    g = G.rmat(scale, 16, 42)
    path = tmp_path / f"rmat{scale}.mtx"
    write_mtx(path, g)
    res = subprocess.run([DROPIN_REF, str(path), "20", "o2"], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr
    assert "dropin_ref" in res.stdout
    # oracle O2 on the reference's own adjacency<1>: the production solver nw::graph::page_rank (v11)
    o2 = dict(kv.split("=") for kv in res.stdout.strip().splitlines()[-1].split()[1:])
    assert float(o2["converged_max_abs"]) <= 1e-7 and int(o2["top100_order_breaks"]) == 0
    assert int(o2["thr_sweeps_engine"]) == int(o2["thr_sweeps_v10"]) and int(o2["thr_sweeps_v11"]) >= 1
