"""The C-ABI libraries load and export every symbol their headers declare
(CPU only: no compute call is made without a GPU)."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT, has_gpu

INCLUDE = os.path.join(ROOT, "include")


def declared_functions(header):
    text = open(os.path.join(INCLUDE, header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:int|void|const char\s*\*)\s+(nw\w+)\s*\(", text, flags=re.M)
    assert names, header
    return sorted(set(names))


@pytest.mark.parametrize("header,lib", [("nwgpu.h", "nwgraph_b200/libnwgpu.so"),
                                        ("nwgraph_gen.h", "nwgraph_b200/libnwgen.so")])
def test_library_exports_header_symbols(header, lib):
    L = C.CDLL(os.path.join(ROOT, lib))
    missing = [n for n in declared_functions(header) if not hasattr(L, n)]
    assert not missing, f"{lib} lacks {missing}"


def test_python_binding_covers_header():
    from nwgraph_b200 import _native as N
    assert set(declared_functions("nwgpu.h")) == set(N.SIGNATURES)
    N.lib()


def test_abi_version():
    from nwgraph_b200 import _native as N
    assert N.lib().nwgpu_abi_version() == 2


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_no_device_fails_loudly():
    """Without a GPU the engine reports NWGPU_ERR_NO_DEVICE; it has no CPU path."""
    import numpy as np
    from nwgraph_b200 import Graph, NwgpuError
    from nwgraph_b200 import _native as N
    with pytest.raises(NwgpuError) as ei:
        Graph(np.array([0, 1, 2], np.uint32), np.array([1, 0], np.uint32))
    assert ei.value.status == N.ERR_NO_DEVICE


def test_null_arguments_rejected_before_device_use():
    from nwgraph_b200 import _native as N
    h = C.c_void_p()
    assert N.lib().nwgpu_graph_create(None, None, None, 3, 0, 0, C.byref(h)) == N.ERR_INVALID_ARG
    assert "row_ptr" in N.last_error()
    assert N.lib().nwgpu_graph_create(None, None, None, 3, 0, 0, None) == N.ERR_INVALID_ARG
    assert N.lib().nwgpu_pr_run(None, None, None, 0.85, 1e-4, 20, None, None) == N.ERR_INVALID_ARG
    assert N.lib().nwgpu_graph_destroy(None) == N.OK


def test_entry_count_limit_rejected_before_device_use():
    """nnz above 2^32 - 512 is refused before any copy: the sweep forms entry indices up to 255 past a row's
    end in 32-bit arithmetic (the reference's own row pointers are uint32, page_rank.hpp:129)."""
    import numpy as np
    from nwgraph_b200 import _native as N
    rp = np.zeros(4, np.uint32)
    cl = np.zeros(4, np.uint32)
    h = C.c_void_p()
    for nnz in (2**32 - 511, 2**32 - 16, 2**32):
        rc = N.lib().nwgpu_graph_create(rp.ctypes.data, cl.ctypes.data, None, 3, nnz, 0, C.byref(h))
        assert rc == N.ERR_INVALID_ARG, nnz
        assert "limit" in N.last_error()
