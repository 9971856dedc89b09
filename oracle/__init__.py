"""CPU oracle for the PageRank hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its cpu_baseline
leg and its ``--impl reference`` arm) may import this package, and only as the
checker or the CPU baseline. The product path (``nwgraph_b200`` and
``libnwgpu.so``) never imports it and has no CPU fallback.

Two libraries sit behind this module:

* ``oracle/liboracle.so`` -- the C restatement in ``oracle/pr_oracle.c``
  (Jacobi ``page_rank_v10``, Gauss-Seidel ``page_rank`` v11 on one thread,
  ``page_rank_v1`` in double, and FP64 oracles for plain / personalized /
  weighted PageRank and the implicit adjoint).
* ``oracle/_ref/libnwref.so`` -- NWGraph's own headers compiled against the
  TBB-API shim (``oracle/ref_driver.cpp``); ``libnwref_fast.so`` is the same at
  the reference's release flags, used for timing. Present only where
  ``make -C oracle ref`` ran (it needs the reference tree), and shipped as a
  built file otherwise.

Parity pins: see ``tests/test_oracle.py`` (restatement == compiled reference,
bit for bit; karate golden vector of test/page_rank_test.cpp:72-75).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_u32p = C.POINTER(C.c_uint32)
_f32p = C.POINTER(C.c_float)
_f64p = C.POINTER(C.c_double)


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def default_reference_root() -> str:
    """Where the reference tree is looked for when NWGRAPH_REF is unset: a
    directory named ``reference`` beside this repository."""
    return os.path.normpath(os.path.join(_HERE, "..", "..", "reference"))


def build(with_reference: bool | None = None) -> None:
    """Compile the restatement (always) and the reference driver (when the
    reference tree is present, or when asked)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    ref_root = os.environ.get("NWGRAPH_REF") or default_reference_root()
    if with_reference is None:
        with_reference = os.path.isdir(os.path.join(ref_root, "include", "nwgraph"))
    if with_reference:
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={ref_root}"], check=True)


_lib = None
_ref = {}


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build(with_reference=False)
        L = C.CDLL(path)
        L.orc_pr_jacobi_f32.restype = C.c_int64
        L.orc_pr_jacobi_f32.argtypes = [_u32p, _u32p, C.c_uint64, _u32p, _f32p, C.c_float, C.c_float, C.c_uint64, _f64p]
        L.orc_pr_gauss_seidel_f32.restype = C.c_int64
        L.orc_pr_gauss_seidel_f32.argtypes = L.orc_pr_jacobi_f32.argtypes
        L.orc_ppr_jacobi_f32.restype = C.c_int64
        L.orc_ppr_jacobi_f32.argtypes = [_u32p, _u32p, C.c_uint64, _u32p, C.c_uint32, _f32p, C.c_float, C.c_float,
                                         C.c_uint64, _f64p]
        L.orc_pr_residual_f32.restype = C.c_int64
        L.orc_pr_residual_f32.argtypes = L.orc_pr_jacobi_f32.argtypes
        L.orc_pr_v1_f64.restype = C.c_int64
        L.orc_pr_v1_f64.argtypes = [_u32p, _u32p, C.c_uint64, _u32p, _f64p, C.c_double, C.c_double, C.c_uint64]
        L.orc_pr_f64.restype = C.c_int64
        L.orc_pr_f64.argtypes = [_u32p, _u32p, C.c_uint64, _f32p, _f64p, _f64p, C.c_double, C.c_double, C.c_uint64,
                                 _f64p, _f64p]
        L.orc_pr_vjp_f64.restype = C.c_int64
        L.orc_pr_vjp_f64.argtypes = [_u32p, _u32p, C.c_uint64, _f32p, _f64p, _f64p, C.c_double, C.c_double, C.c_uint64,
                                     _f64p, _f64p, _f64p]
        _lib = L
    return _lib


def ref_available(fast: bool = False) -> bool:
    name = "libnwref_fast.so" if fast else "libnwref.so"
    return os.path.exists(os.path.join(_HERE, "_ref", name))


def ref(fast: bool = False):
    """NWGraph's own page_rank compiled from its headers (oracle/_ref)."""
    key = "fast" if fast else "exact"
    if key not in _ref:
        path = os.path.join(_HERE, "_ref", "libnwref_fast.so" if fast else "libnwref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (make -C oracle ref needs the reference tree)")
        L = C.CDLL(path)
        L.nwref_page_rank_f32.restype = C.c_int
        L.nwref_page_rank_f32.argtypes = [C.c_int, _u32p, _u32p, C.c_uint64, _u32p, _f32p, C.c_float, C.c_float,
                                          C.c_uint64, C.c_int, _f64p, _f64p, C.c_int]
        L.nwref_page_rank_v1_f64.restype = C.c_int
        L.nwref_page_rank_v1_f64.argtypes = [_u32p, _u32p, C.c_uint64, _u32p, _f64p, C.c_double, C.c_double,
                                             C.c_uint64]
        L.nwref_build_degrees.restype = C.c_int
        L.nwref_build_degrees.argtypes = [_u32p, _u32p, C.c_uint64, _u32p, C.c_int]
        L.nwref_fill_adj1.restype = C.c_int
        L.nwref_fill_adj1.argtypes = [_u32p, _u32p, C.c_uint64, C.c_uint64, _u32p, _u32p]
        L.nwref_read_mm_edges.restype = C.c_int
        L.nwref_read_mm_edges.argtypes = [C.c_char_p, _u32p, _u32p, C.c_uint64, C.POINTER(C.c_uint64),
                                          C.POINTER(C.c_uint64)]
        L.nwref_read_nw_edges.restype = C.c_int
        L.nwref_read_nw_edges.argtypes = L.nwref_read_mm_edges.argtypes
        L.nwref_write_nw_edges.restype = C.c_int
        L.nwref_write_nw_edges.argtypes = [C.c_char_p, _u32p, _u32p, C.c_uint64, C.c_uint64]
        L.nwref_write_adj1.restype = C.c_int
        L.nwref_write_adj1.argtypes = [C.c_char_p, _u32p, _u32p, C.c_uint64]
        L.nwref_build_csr.restype = C.c_int
        L.nwref_build_csr.argtypes = [_u32p, _u32p, C.c_uint64, C.c_uint64, C.c_int, _u32p, _u32p, C.c_uint64,
                                      C.POINTER(C.c_uint64)]
        L.nwref_load_mm.restype = C.c_void_p
        L.nwref_load_mm.argtypes = [C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.nwref_copy_csr.restype = None
        L.nwref_copy_csr.argtypes = [C.c_void_p, _u32p, _u32p]
        L.nwref_free.restype = None
        L.nwref_free.argtypes = [C.c_void_p]
        L.nwref_graph_create.restype = C.c_void_p
        L.nwref_graph_create.argtypes = [_u32p, _u32p, C.c_uint64, _u32p]
        L.nwref_graph_destroy.restype = None
        L.nwref_graph_destroy.argtypes = [C.c_void_p]
        L.nwref_graph_page_rank_f32.restype = C.c_int
        L.nwref_graph_page_rank_f32.argtypes = [C.c_void_p, C.c_int, _f32p, C.c_float, C.c_float, C.c_uint64, C.c_int,
                                                _f64p, _f64p, C.c_int]
        _ref[key] = L
    return _ref[key]


# --------------------------------------------------------------------------
# restatement (oracle/pr_oracle.c)
# --------------------------------------------------------------------------

def out_degree(row_ptr, col, n):
    """Out-degree per vertex from an adjacency<1> CSR (bench/gapbs/common.hpp:110-121)."""
    return np.bincount(np.asarray(col, dtype=np.int64), minlength=int(n)).astype(np.uint32)


def jacobi_f32(row_ptr, col, deg, damping=0.85, threshold=1e-4, max_iters=20):
    """page_rank_v10 restated. Returns (ranks float32, sweeps, errors)."""
    n = len(row_ptr) - 1
    r = np.empty(n, np.float32)
    errs = np.zeros(max(int(max_iters), 1), np.float64)
    it = lib().orc_pr_jacobi_f32(_p(row_ptr, _u32p), _p(col, _u32p), n, _p(deg, _u32p), _p(r, _f32p), damping,
                                 threshold, int(max_iters), _p(errs, _f64p))
    return r, int(it), errs[: int(it)]


def ppr_jacobi_f32(row_ptr, col, deg, seed, damping=0.85, threshold=1e-6, max_iters=100):
    """Personalised FP32 Jacobi (one-hot teleport at seed). Returns (ranks, sweeps, errors)."""
    n = len(row_ptr) - 1
    r = np.empty(n, np.float32)
    errs = np.zeros(max(int(max_iters), 1), np.float64)
    it = lib().orc_ppr_jacobi_f32(_p(row_ptr, _u32p), _p(col, _u32p), n, _p(deg, _u32p), int(seed), _p(r, _f32p),
                                  damping, threshold, int(max_iters), _p(errs, _f64p))
    return r, int(it), errs[: int(it)]


def residual_f32(row_ptr, col, deg, damping=0.85, threshold=1e-4, max_iters=20):
    """page_rank_v13 (residual push) restated. Returns (ranks, iterations, pushes per iteration)."""
    n = len(row_ptr) - 1
    r = np.empty(n, np.float32)
    cnt = np.zeros(max(int(max_iters), 1), np.float64)
    it = lib().orc_pr_residual_f32(_p(row_ptr, _u32p), _p(col, _u32p), n, _p(deg, _u32p), _p(r, _f32p), damping,
                                   threshold, int(max_iters), _p(cnt, _f64p))
    return r, int(it), cnt[: int(it)]


def gauss_seidel_f32(row_ptr, col, deg, damping=0.85, threshold=1e-4, max_iters=20):
    """page_rank (v11) on one thread, restated."""
    n = len(row_ptr) - 1
    r = np.empty(n, np.float32)
    errs = np.zeros(max(int(max_iters), 1), np.float64)
    it = lib().orc_pr_gauss_seidel_f32(_p(row_ptr, _u32p), _p(col, _u32p), n, _p(deg, _u32p), _p(r, _f32p), damping,
                                       threshold, int(max_iters), _p(errs, _f64p))
    return r, int(it), errs[: int(it)]


def v1_f64(row_ptr, col, deg, damping=0.85, threshold=1e-4, max_iters=100):
    n = len(row_ptr) - 1
    r = np.empty(n, np.float64)
    it = lib().orc_pr_v1_f64(_p(row_ptr, _u32p), _p(col, _u32p), n, _p(deg, _u32p), _p(r, _f64p), damping,
                             threshold, int(max_iters))
    return r, int(it)


def pr_f64(row_ptr, col, weights=None, teleport=None, r0=None, damping=0.85, tol=1e-14, max_iters=10000):
    """FP64 Jacobi power iteration, leak semantics (oracles O3/O4)."""
    n = len(row_ptr) - 1
    r = np.empty(n, np.float64)
    fe = np.zeros(1, np.float64)
    w = None if weights is None else np.ascontiguousarray(weights, np.float32)
    t = None if teleport is None else np.ascontiguousarray(teleport, np.float64)
    x0 = None if r0 is None else np.ascontiguousarray(r0, np.float64)
    it = lib().orc_pr_f64(_p(row_ptr, _u32p), _p(col, _u32p), n, _p(w, _f32p), _p(t, _f64p), _p(x0, _f64p), damping,
                          tol, int(max_iters), _p(r, _f64p), _p(fe, _f64p))
    return r, int(it), float(fe[0])


def vjp_f64(row_ptr, col, r, cvec, weights=None, damping=0.85, tol=1e-14, max_iters=10000, want_dw=True):
    """Implicit adjoint of the fixed point. Returns (lambda, dL/dt, dL/dw)."""
    n = len(row_ptr) - 1
    nnz = int(row_ptr[-1])
    lam = np.empty(n, np.float64)
    dt = np.empty(n, np.float64)
    dw = np.empty(nnz, np.float64) if want_dw else None
    w = None if weights is None else np.ascontiguousarray(weights, np.float32)
    lib().orc_pr_vjp_f64(_p(row_ptr, _u32p), _p(col, _u32p), n, _p(w, _f32p),
                         _p(np.ascontiguousarray(r, np.float64), _f64p), _p(np.ascontiguousarray(cvec, np.float64), _f64p),
                         damping, tol, int(max_iters), _p(lam, _f64p), _p(dt, _f64p), _p(dw, _f64p))
    return lam, dt, dw


# --------------------------------------------------------------------------
# NWGraph itself (oracle/_ref)
# --------------------------------------------------------------------------

def ref_page_rank(version, row_ptr, col, deg, damping=0.85, threshold=1e-4, max_iters=20, nthreads=1, fast=False):
    """Run nw::graph::page_rank (11), page_rank_v10 (10) or page_rank_v1 (1)
    from the reference headers. Returns (ranks, sweeps, errors, seconds per sweep)."""
    n = len(row_ptr) - 1
    r = np.empty(n, np.float32)
    rows = max(int(max_iters), 1)
    errs = np.zeros(rows, np.float64)
    secs = np.zeros(rows, np.float64)
    it = ref(fast).nwref_page_rank_f32(version, _p(row_ptr, _u32p), _p(col, _u32p), n, _p(deg, _u32p), _p(r, _f32p),
                                       damping, threshold, int(max_iters), int(nthreads), _p(errs, _f64p),
                                       _p(secs, _f64p), rows)
    if it < 0:
        raise ValueError(f"unknown page_rank version {version}")
    k = min(it, rows)
    return r, int(it), errs[:k], secs[:k]


class RefGraph:
    """NWGraph adjacency<1> + degrees held in the reference library, for
    repeated timing runs of its page_rank without re-copying the CSR."""

    def __init__(self, row_ptr, col, deg, fast=True):
        self.n = len(row_ptr) - 1
        self._L = ref(fast)
        self._h = self._L.nwref_graph_create(_p(row_ptr, _u32p), _p(col, _u32p), self.n, _p(deg, _u32p))

    def page_rank(self, version=11, damping=0.85, threshold=0.0, max_iters=2, nthreads=1):
        r = np.empty(self.n, np.float32)
        rows = max(int(max_iters), 1)
        errs = np.zeros(rows, np.float64)
        secs = np.zeros(rows, np.float64)
        it = self._L.nwref_graph_page_rank_f32(self._h, version, _p(r, _f32p), damping, threshold, int(max_iters),
                                               int(nthreads), _p(errs, _f64p), _p(secs, _f64p), rows)
        if it < 0:
            raise ValueError(f"unknown page_rank version {version}")
        k = min(it, rows)
        return r, int(it), errs[:k], secs[:k]

    def close(self):
        if self._h:
            self._L.nwref_graph_destroy(self._h)
            self._h = None

    __del__ = close


class _NwgenCsr(C.Structure):
    _fields_ = [("n", C.c_uint64), ("nnz", C.c_uint64), ("row_ptr", _u32p), ("col", _u32p)]


def ref_rmat(scale, edge_factor=16, seed=42, abc=(0.57, 0.19, 0.19), nthreads=0):
    """The benchmark's seeded RMAT CSR (symmetrised, deduplicated, rows
    sorted), built by the copy of the input builder that
    oracle/_ref/libnwref_fast.so carries, so that a process timing NWGraph
    maps no library of the engine. The same graph bit for bit as
    nwgraph_b200.graphs.rmat. Returns (row_ptr, col)."""
    L = ref(fast=True)
    if not getattr(L, "_nwgen_bound", False):
        L.nwgen_rmat.restype = C.c_int
        L.nwgen_rmat.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int,
                                 C.POINTER(_NwgenCsr)]
        L.nwgen_free.restype = None
        L.nwgen_free.argtypes = [C.POINTER(_NwgenCsr)]
        L._nwgen_bound = True
    g = _NwgenCsr()
    rc = L.nwgen_rmat(int(scale), float(edge_factor), abc[0], abc[1], abc[2], int(seed), int(nthreads), C.byref(g))
    if rc != 0:
        raise RuntimeError(f"nwgen_rmat failed with status {rc}")
    try:
        n, nnz = int(g.n), int(g.nnz)
        rp = np.ctypeslib.as_array(g.row_ptr, shape=(n + 1,)).copy()
        cl = np.ctypeslib.as_array(g.col, shape=(max(nnz, 1),))[:nnz].copy()
    finally:
        L.nwgen_free(C.byref(g))
    return rp, cl


def ref_page_rank_v1_f64(row_ptr, col, deg, damping=0.85, threshold=1e-7, max_iters=100):
    n = len(row_ptr) - 1
    r = np.empty(n, np.float64)
    ref().nwref_page_rank_v1_f64(_p(row_ptr, _u32p), _p(col, _u32p), n, _p(deg, _u32p), _p(r, _f64p), damping,
                                 threshold, int(max_iters))
    return r


def ref_build_degrees(row_ptr, col, nthreads=1):
    n = len(row_ptr) - 1
    d = np.empty(n, np.uint32)
    ref().nwref_build_degrees(_p(row_ptr, _u32p), _p(col, _u32p), n, _p(d, _u32p), int(nthreads))
    return d


def ref_fill_adj1(src, dst, n):
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    m = len(src)
    rp = np.empty(int(n) + 1, np.uint32)
    cl = np.empty(max(m, 1), np.uint32)
    rc = ref().nwref_fill_adj1(_p(src, _u32p), _p(dst, _u32p), m, int(n), _p(rp, _u32p), _p(cl, _u32p))
    if rc != 0:
        raise RuntimeError("nwref_fill_adj1 failed")
    return rp, cl[:m]


# Flags of the edge-list -> CSR build (the values of include/nwgpu.h's NWGPU_EDGES_*).
BY_SOURCE, UNDIRECTED, REMOVE_SELF_LOOPS, UNIQUE, UNIQUE_ENTRIES = 0x2, 0x4, 0x8, 0x10, 0x20


def build_csr(src, dst, n, flags):
    """Edge list -> CSR restated: the reference's remove_self_loops
    (build.hpp:404-410), lexical sort + uniq on the edge list (:58-69,
    :394-402) and fill_directed / fill_undirected (:209-272) with
    sort_adjacency (:311-321), i.e. rows indexed by target (by source with
    BY_SOURCE), both directions of every edge with UNDIRECTED, rows sorted.
    UNIQUE_ENTRIES then drops repeated (row, col) entries of the result (the
    host builder's simple-graph clean-up, graphgen.cpp; not a reference step).
    Returns (row_ptr, col, degrees) with degrees = column occurrences
    (bench/gapbs/common.hpp:110-121)."""
    s = np.asarray(src, np.uint64)
    d = np.asarray(dst, np.uint64)
    if flags & REMOVE_SELF_LOOPS:
        keep = s != d
        s, d = s[keep], d[keep]
    if flags & UNIQUE:
        pairs = np.unique(s << np.uint64(32) | d)
        s, d = pairs >> np.uint64(32), pairs & np.uint64(0xFFFFFFFF)
    row, col = (s, d) if flags & BY_SOURCE else (d, s)
    if flags & UNDIRECTED:
        row, col = np.concatenate([row, col]), np.concatenate([col, row])
    keys = np.sort(row << np.uint64(32) | col)
    if flags & UNIQUE_ENTRIES:
        keys = np.unique(keys)
    r = (keys >> np.uint64(32)).astype(np.int64)
    c = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    rp = np.zeros(int(n) + 1, np.uint32)
    rp[1:] = np.cumsum(np.bincount(r, minlength=int(n)))
    return rp, c, np.bincount(c, minlength=int(n)).astype(np.uint32)


def ref_build_csr(src, dst, n, flags):
    """The same through the reference's own code (oracle/_ref); (row_ptr, col).
    UNIQUE_ENTRIES is not a reference step and is refused."""
    if flags & UNIQUE_ENTRIES:
        raise ValueError("UNIQUE_ENTRIES has no reference counterpart")
    flags = ((1 if flags & BY_SOURCE else 0) | (2 if flags & UNDIRECTED else 0) | (4 if flags & REMOVE_SELF_LOOPS else 0)
             | (8 if flags & UNIQUE else 0))
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    m = len(src)
    cap = 2 * m + 1
    rp = np.empty(int(n) + 1, np.uint32)
    cl = np.empty(cap, np.uint32)
    nnz = C.c_uint64()
    if ref().nwref_build_csr(_p(src, _u32p), _p(dst, _u32p), m, int(n), int(flags), _p(rp, _u32p), _p(cl, _u32p), cap,
                             C.byref(nnz)) != 0:
        raise RuntimeError("nwref_build_csr failed")
    return rp, cl[: nnz.value]


def _ref_edges(fn, path, cap):
    src = np.empty(max(cap, 1), np.uint32)
    dst = np.empty(max(cap, 1), np.uint32)
    m, n = C.c_uint64(), C.c_uint64()
    if fn(path.encode(), _p(src, _u32p), _p(dst, _u32p), cap, C.byref(m), C.byref(n)) != 0:
        raise RuntimeError("reference edge reader failed")
    return src[: m.value].copy(), dst[: m.value].copy(), int(n.value)


def ref_read_mm_edges(path, cap):
    """The edge list NWGraph's read_mm<directed> builds (oracle/_ref): (src, dst, n)."""
    return _ref_edges(ref().nwref_read_mm_edges, path, cap)


def ref_read_nw_edges(path, cap):
    """The edge list NWGraph's edge_list::deserialize reads (oracle/_ref): (src, dst, n)."""
    return _ref_edges(ref().nwref_read_nw_edges, path, cap)


def ref_write_nw_edges(path, src, dst, n):
    """NWGraph's edge_list::serialize of the edges (oracle/_ref)."""
    s = np.ascontiguousarray(src, np.uint32)
    d = np.ascontiguousarray(dst, np.uint32)
    if ref().nwref_write_nw_edges(path.encode(), _p(s, _u32p), _p(d, _u32p), len(s), int(n)) != 0:
        raise RuntimeError("nwref_write_nw_edges failed")


def ref_write_adj1(path, row_ptr, col):
    """NWGraph's adjacency<1>::serialize of the CSR (oracle/_ref)."""
    rp = np.ascontiguousarray(row_ptr, np.uint32)
    cl = np.ascontiguousarray(col, np.uint32)
    if ref().nwref_write_adj1(path.encode(), _p(rp, _u32p), _p(cl, _u32p), len(rp) - 1) != 0:
        raise RuntimeError("nwref_write_adj1 failed")


def ref_load_mm(path):
    n = C.c_uint64()
    nnz = C.c_uint64()
    h = ref().nwref_load_mm(path.encode(), C.byref(n), C.byref(nnz))
    rp = np.empty(n.value + 1, np.uint32)
    cl = np.empty(max(nnz.value, 1), np.uint32)
    ref().nwref_copy_csr(h, _p(rp, _u32p), _p(cl, _u32p))
    ref().nwref_free(h)
    return rp, cl[: nnz.value]
