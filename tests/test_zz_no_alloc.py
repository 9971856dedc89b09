"""nwgpu_pr_run_noalloc: PageRank with no allocation, through the C ABI.

The entry point has no counterpart in the reference. Its output is compared
with nwgpu_pr_run's (the handle-based entry point) on the same graph, within
the parity tolerance used for the engine, on two calls in a row. The file is
named so that pytest collects it last: it must pass both in a fresh process
(the first call on the device looks up the static working array) and after
every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from nwgraph_b200 import Graph, graphs as G
from nwgraph_b200 import _native as N

pytestmark = pytest.mark.gpu

MAX_ABS = 1e-6
L1 = 1e-5


def close(a, b):
    d = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))
    assert d.max() <= MAX_ABS, f"max-abs {d.max():.3e}"
    assert d.sum() <= L1, f"L1 {d.sum():.3e}"


def last_error():
    buf = C.create_string_buffer(512)
    N.lib().nwgpu_last_error(buf, 512)
    return buf.value.decode()


def noalloc(rp, cl, n, nnz, dg, out, d, thr, iters, stream=None, errors_cap=0):
    st = N.PrStats()
    errs = None
    if errors_cap:
        errs = np.zeros(errors_cap, np.float64)
        st.errors = errs.ctypes.data_as(C.POINTER(C.c_double))
        st.errors_cap = errors_cap
    rc = N.lib().nwgpu_pr_run_noalloc(rp, cl, n, nnz, dg, out, d, thr, iters, stream, C.byref(st))
    return rc, st, errs


@pytest.fixture(scope="module")
def cases():
    return [("rmat12", G.rmat(12, 16, 3)), ("rmat16", G.rmat(16, 16, 8)), ("grid", G.grid(60_000))]


@pytest.mark.parametrize("thr,iters", [(0.0, 20), (1e-6, 100)])
def test_noalloc_matches_pr_run(gpu, cases, thr, iters):
    import torch
    dev = torch.device("cuda")
    for name, g in cases:
        deg = g.out_degree()
        ref = np.empty(g.n, np.float32)
        with Graph(g.row_ptr, g.col) as h:
            ref_st = h.page_rank(deg, ref, 0.85, thr, iters, record_errors=True)
        rp = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
        cl = torch.from_numpy(g.col.view(np.int32)).to(dev)
        dg = torch.from_numpy(deg.view(np.int32)).to(dev)
        outs = []
        for call in range(2):
            out = torch.full((g.n,), -1.0, dtype=torch.float32, device=dev)
            torch.cuda.synchronize()
            rc, st, errs = noalloc(rp.data_ptr(), cl.data_ptr(), g.n, g.nnz, dg.data_ptr(), out.data_ptr(), 0.85, thr,
                                   iters, errors_cap=iters)
            assert rc == N.OK, f"{name} call {call}: {last_error()}"
            got = out.cpu().numpy()
            close(got, ref)
            if thr == 0.0:
                assert st.iterations == iters and not st.converged
            else:
                # the stopping sweep: FP64 sums of the same FP32 changes in another order may differ at a tie
                assert abs(int(st.iterations) - int(ref_st.iterations)) <= 1 and st.converged
            m = int(st.iterations)
            k = min(m, int(ref_st.iterations))
            assert np.allclose(errs[:k], ref_st.errors[:k], rtol=1e-4, atol=1e-6)
            assert st.final_error == errs[m - 1]
            outs.append(got)
        assert np.array_equal(outs[0], outs[1]), f"{name}: two no-alloc calls in a row differ"


def test_noalloc_matches_oracle_and_stream(gpu):
    import torch
    g = G.rmat(13, 16, 21)
    deg = g.out_degree()
    ref, _, _ = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 15)
    dev = torch.device("cuda")
    rp = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    cl = torch.from_numpy(g.col.view(np.int32)).to(dev)
    dg = torch.from_numpy(deg.view(np.int32)).to(dev)
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    for _ in range(2):
        out = torch.empty(g.n, dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        rc, st, _ = noalloc(rp.data_ptr(), cl.data_ptr(), g.n, g.nnz, dg.data_ptr(), out.data_ptr(), 0.85, 0.0, 15,
                            stream=s.cuda_stream)
        assert rc == N.OK, last_error()
        assert st.iterations == 15
        close(out.cpu().numpy(), ref)


def test_noalloc_rejects(gpu):
    import torch
    g = G.rmat(10, 8, 2)
    deg = g.out_degree()
    dev = torch.device("cuda")
    rp = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    cl = torch.from_numpy(g.col.view(np.int32)).to(dev)
    dg = torch.from_numpy(deg.view(np.int32)).to(dev)
    out = torch.empty(g.n + 8, dtype=torch.float32, device=dev)
    args = (0.85, 0.0, 5)
    # beyond the static working array: rejected before any device work
    rc, _, _ = noalloc(rp.data_ptr(), cl.data_ptr(), N.NOALLOC_MAX_VERTICES + 1, g.nnz, dg.data_ptr(), out.data_ptr(),
                       *args)
    assert rc == N.ERR_INVALID_ARG and "no-alloc limit" in last_error()
    rc, _, _ = noalloc(rp.data_ptr(), cl.data_ptr(), g.n, N.NOALLOC_MAX_ENTRIES + 1, dg.data_ptr(), out.data_ptr(),
                       *args)
    assert rc == N.ERR_INVALID_ARG and "no-alloc limit" in last_error()
    # misaligned output, host memory instead of device memory
    rc, _, _ = noalloc(rp.data_ptr(), cl.data_ptr(), g.n, g.nnz, dg.data_ptr(), out.data_ptr() + 4, *args)
    assert rc == N.ERR_INVALID_ARG and "16-byte aligned" in last_error()
    host_deg = np.zeros(g.n + 16, np.uint32)
    p = host_deg.ctypes.data
    p += (-p) % 16
    rc, _, _ = noalloc(rp.data_ptr(), cl.data_ptr(), g.n, g.nnz, p, out.data_ptr(), *args)
    assert rc == N.ERR_INVALID_ARG and "device memory" in last_error()
    # a column index out of range is caught by the on-device validation
    bad = g.col.copy()
    bad[len(bad) // 2] = g.n + 5
    cb = torch.from_numpy(bad.view(np.int32)).to(dev)
    rc, _, _ = noalloc(rp.data_ptr(), cb.data_ptr(), g.n, g.nnz, dg.data_ptr(), out.data_ptr(), *args)
    assert rc == N.ERR_INVALID_GRAPH and "col index" in last_error()
    # the engine is still usable afterwards
    rc, st, _ = noalloc(rp.data_ptr(), cl.data_ptr(), g.n, g.nnz, dg.data_ptr(), out.data_ptr(), *args)
    assert rc == N.OK and st.iterations == 5


def _cudart():
    import os
    import nvidia.cuda_runtime as cr
    lib = C.CDLL(os.path.join(list(cr.__path__)[0], "lib", "libcudart.so.12"))
    lib.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    lib.cudaFree.argtypes = [C.c_void_p]
    lib.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    return lib


def _random_graph(n, m):
    rng = np.random.default_rng(n + m)
    return G.from_edges(rng.integers(0, n, m), rng.integers(0, n, m), n, symmetrize=False)


# (n, sampled edges, expected nnz): n and nnz cover every residue mod 4, so row_ptr (n + 1 elements), col (nnz),
# degrees and ranks (n) each end at every position inside their final 16-byte word in some case
@pytest.mark.parametrize("n,m,nnz", [(3001, 20_011, 19_991), (3002, 15_003, 14_985), (3003, 30_003, 29_946),
                                     (4096, 40_000, 39_963), (3001, 20_012, 19_984)])
def test_noalloc_arrays_at_allocation_end(gpu, n, m, nnz):
    """Every array is placed at the end of its own cudaMalloc of a 2 MiB multiple: it starts at the last
    16-byte-aligned offset it fits at, so it ends inside the allocation's final 16 bytes (exactly at the end when
    its byte length is a multiple of 16). The solve reads nothing past the arrays' lengths, and its ranks equal
    the handle entry point's and the oracle's."""
    import torch
    g = _random_graph(n, m)
    assert g.nnz == nnz
    deg = g.out_degree()
    ref, _, _ = O.jacobi_f32(g.row_ptr, g.col, deg, 0.85, 0.0, 12)
    rt = _cudart()
    two_mib = 2 << 20
    allocs, ptrs = [], {}
    try:
        for key, arr in (("row_ptr", g.row_ptr), ("col", g.col), ("deg", deg), ("ranks", np.zeros(g.n, np.float32))):
            nbytes = arr.nbytes
            size = (nbytes + 16 + two_mib - 1) // two_mib * two_mib
            base = C.c_void_p()
            assert rt.cudaMalloc(C.byref(base), size) == 0
            allocs.append(base.value)
            off = (size - nbytes) & ~15
            assert off + nbytes <= size and size - (off + nbytes) < 16
            p = base.value + off
            assert rt.cudaMemcpy(p, arr.ctypes.data, nbytes, 1) == 0
            ptrs[key] = p
        torch.cuda.synchronize()
        outs = []
        for _ in range(2):
            rc, st, _ = noalloc(ptrs["row_ptr"], ptrs["col"], g.n, g.nnz, ptrs["deg"], ptrs["ranks"], 0.85, 0.0, 12)
            assert rc == N.OK, last_error()
            assert st.iterations == 12
            got = np.empty(g.n, np.float32)
            assert rt.cudaMemcpy(got.ctypes.data, ptrs["ranks"], got.nbytes, 2) == 0
            close(got, ref)
            outs.append(got)
        assert np.array_equal(outs[0], outs[1])
        handle_out = np.empty(g.n, np.float32)
        with Graph(g.row_ptr, g.col) as h:
            h.page_rank(deg, handle_out, 0.85, 0.0, 12)
        close(outs[0], handle_out)
    finally:
        torch.cuda.synchronize()
        for p in allocs:
            rt.cudaFree(p)
