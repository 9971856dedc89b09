"""The extensions on the reference's own test matrices (test/data/*.mtx, as its
driver loads them: tests/golden/refdata.npz).

* batched personalised PageRank (nwgpu_ppr_batched), each column against the
  oracle's FP32 restatement of the single-seed solve (oracle.ppr_jacobi_f32)
  at a fixed sweep count: 1e-6 max-abs, 1e-5 L1;
* residual-push PageRank (nwgpu_pr_residual_run) against page_rank_v13
  restated (oracle.residual_f32, bit-exact with the compiled reference) with
  every residual pushed (threshold 0): ranks to 1e-5 relative (v13's ranks
  are unnormalised and its sums serial), push counts per iteration equal.
"""
import numpy as np
import pytest

import oracle as O
from conftest import REFDATA_NAMES
from nwgraph_b200 import Graph

pytestmark = pytest.mark.gpu

D = 0.85


@pytest.mark.parametrize("name", REFDATA_NAMES)
def test_batched_ppr_on_reference_matrices(gpu, refdata, name):
    g = refdata[name]
    rp, cl, deg = g["row_ptr"], g["col"], g["deg"]
    n = len(rp) - 1
    seeds = np.unique(np.linspace(0, n - 1, min(n, 8)).astype(np.uint32))
    out = np.empty((n, len(seeds)), np.float32)
    with Graph(rp, cl) as h:
        st = h.ppr_batched(deg, seeds, out, D, 0.0, 15)
    assert st.iterations == 15
    for c, s in enumerate(seeds):
        ref, it, _ = O.ppr_jacobi_f32(rp, cl, deg, int(s), D, 0.0, 15)
        d = np.abs(out[:, c].astype(np.float64) - ref)
        assert it == 15 and d.max() <= 1e-6 and d.sum() <= 1e-5, (name, int(s), d.max())


@pytest.mark.parametrize("name", REFDATA_NAMES)
def test_residual_push_on_reference_matrices(gpu, refdata, name):
    g = refdata[name]
    rp, cl, deg = g["row_ptr"], g["col"], g["deg"]
    n = len(rp) - 1
    with Graph(rp, cl) as h:
        out = np.empty(n, np.float32)
        st = h.page_rank_residual(deg, out, D, 0.0, 10, record_errors=True)
    ref, it, cnt = O.residual_f32(rp, cl, deg, D, 0.0, 10)
    assert st.iterations == it
    assert np.array_equal(np.asarray(st.errors), cnt)
    scale = np.maximum(np.abs(ref.astype(np.float64)), 1e-3)
    assert np.max(np.abs(out.astype(np.float64) - ref) / scale) <= 1e-5, name
