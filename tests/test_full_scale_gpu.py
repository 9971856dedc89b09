"""Parity at the benchmark's full size: RMAT scale 24, edge factor 16
(n = 16,777,216, nnz = 520,771,744), built on the GPU (the same CSR as the
host builder, tests/test_construct_gpu.py).

* the benchmark's solve, 20 fixed sweeps, against page_rank_v10 restated
  (oracle.jacobi_f32, pinned to the reference in test_oracle.py): within 1e-6
  max-abs and 1e-5 L1, per-sweep errors within 1e-6, and the same top-100
  order apart from ties inside 1e-6;
* a size-independent property of every sweep: with leak semantics the new
  ranks sum to (1 - d) + d * (the old ranks of vertices with out-degree > 0),
  checked between the 19th and 20th sweeps in FP64 to 1e-6 relative;
* the 20-sweep ranks are bitwise reproducible.
"""
import numpy as np
import pytest

import oracle as O
from nwgraph_b200 import Graph, construct as K

pytestmark = pytest.mark.gpu

D = 0.85


@pytest.fixture(scope="module")
def rmat24():
    g = K.rmat(24, 16, 42)
    return g, g.out_degree()


def solve(h, deg, sweeps):
    out = np.empty(h.n, np.float32)
    h.page_rank(deg, out, D, 0.0, sweeps)
    return out


def test_twenty_sweeps_match_page_rank_v10(gpu, rmat24):
    g, deg = rmat24
    assert g.nnz == 520_771_744
    with Graph(g.row_ptr, g.col) as h:
        r = np.empty(g.n, np.float32)
        st = h.page_rank(deg, r, D, 0.0, 20, record_errors=True)
    ref, it, errs = O.jacobi_f32(g.row_ptr, g.col, deg, D, 0.0, 20)
    d = np.abs(r.astype(np.float64) - ref)
    assert it == 20 and d.max() <= 1e-6 and d.sum() <= 1e-5, (d.max(), d.sum())
    assert np.allclose(st.errors, errs, rtol=1e-4, atol=1e-6)
    top_r = np.argsort(-ref.astype(np.float64), kind="stable")[:100]
    top_g = np.argsort(-r.astype(np.float64), kind="stable")[:100]
    for a, b in zip(top_r, top_g):
        assert a == b or abs(float(ref[a]) - float(ref[b])) <= 1e-6


def test_leak_conservation_and_reproducibility(gpu, rmat24):
    g, deg = rmat24
    with Graph(g.row_ptr, g.col) as h:
        r19 = solve(h, deg, 19)
        r20 = solve(h, deg, 20)
        again = solve(h, deg, 20)
    assert np.array_equal(r20.view(np.uint32), again.view(np.uint32))
    lhs = r20.astype(np.float64).sum()
    rhs = (1.0 - D) + D * r19.astype(np.float64)[deg > 0].sum()
    assert abs(lhs - rhs) <= 1e-6 * rhs, (lhs, rhs)
