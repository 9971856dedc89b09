"""The engine's bounded device waits give up and report it, without a fault.

The merge-path sweeps wait on shared-memory barriers for their bulk copies;
each wait gives up after 2^20 polls and records a fault word that ends the
solve with NWGPU_ERR_CUDA. nwgpu_selftest_bounded_wait runs that same wait loop
on a barrier that nothing ever completes (a flag nobody sets): the wait must
give up, quickly for a small poll count, and the context must stay usable.
"""
import ctypes as C

import numpy as np
import pytest

from nwgraph_b200 import Graph, NwgpuError, graphs as G
from nwgraph_b200 import _native as N

pytestmark = pytest.mark.gpu


def selftest(polls):
    gave_up, ms = C.c_uint32(), C.c_double()
    N.check(N.lib().nwgpu_selftest_bounded_wait(polls, C.byref(gave_up), C.byref(ms)))
    return gave_up.value, ms.value


@pytest.mark.parametrize("polls", [1, 1 << 10, 1 << 14])
def test_wait_gives_up_and_the_context_stays_usable(gpu, polls):
    gave_up, ms = selftest(polls)
    assert gave_up == 1
    assert 0.0 <= ms < 60_000.0
    g = G.rmat(10, 16, 3)  # a solve on the same context afterwards
    with Graph(g.row_ptr, g.col, relabel=False) as h:  # the merge-path sweep, which uses these waits
        r = np.empty(g.n, np.float32)
        st = h.page_rank(g.out_degree(), r, 0.85, 0.0, 5)
    assert st.iterations == 5 and np.isfinite(r).all()


def test_bad_arguments(gpu):
    gave_up, ms = C.c_uint32(), C.c_double()
    for polls in (0, (1 << 20) + 1):
        with pytest.raises(NwgpuError) as ei:
            N.check(N.lib().nwgpu_selftest_bounded_wait(polls, C.byref(gave_up), C.byref(ms)))
        assert ei.value.status == N.ERR_INVALID_ARG
