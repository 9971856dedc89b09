"""Seeded synthetic inputs for the PageRank engine (host side).

Wraps ``libnwgen.so`` (``csrc/graphgen.cpp``, C ABI in ``include/nwgraph_gen.h``)
and adds the small seeded vectors the workloads need (PPR seeds, edge weights,
loss coefficients). Every CSR here is NWGraph's ``adjacency<1>`` layout:
``row_ptr`` = ``indices_`` (n+1 uint32), ``col`` = ``std::get<0>(to_be_indexed_)``
(nnz uint32), row i = in-neighbours of i (include/nwgraph/adjacency.hpp:86-195).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

# RMAT quadrant probabilities used throughout (a, b, c; d = 0.05).
RMAT_ABC = (0.57, 0.19, 0.19)


class _Csr(C.Structure):
    _fields_ = [("n", C.c_uint64), ("nnz", C.c_uint64), ("row_ptr", C.POINTER(C.c_uint32)),
                ("col", C.POINTER(C.c_uint32))]


_gen = None


def _lib():
    global _gen
    if _gen is None:
        path = os.path.join(_HERE, "libnwgen.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run __graft_entry__.build() (nwgraph_b200.build)")
        L = C.CDLL(path)
        L.nwgen_rmat.restype = C.c_int
        L.nwgen_rmat.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int,
                                 C.POINTER(_Csr)]
        L.nwgen_grid.restype = C.c_int
        L.nwgen_grid.argtypes = [C.c_uint64, C.POINTER(_Csr)]
        L.nwgen_from_edges.restype = C.c_int
        L.nwgen_from_edges.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_uint64, C.c_uint64, C.c_int,
                                       C.c_int, C.POINTER(_Csr)]
        L.nwgen_free.restype = None
        L.nwgen_free.argtypes = [C.POINTER(_Csr)]
        _gen = L
    return _gen


@dataclass
class CSR:
    """A compressed adjacency<1>: row i lists the in-neighbours of vertex i."""
    row_ptr: np.ndarray  # uint32[n+1]
    col: np.ndarray      # uint32[nnz]

    @property
    def n(self) -> int:
        return len(self.row_ptr) - 1

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])

    def out_degree(self) -> np.ndarray:
        """Out-degree per vertex (what bench/gapbs/common.hpp:110-121 computes)."""
        return np.bincount(self.col, minlength=self.n).astype(np.uint32)


def _take(rc: int, g: _Csr, what: str) -> CSR:
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")
    try:
        n, nnz = int(g.n), int(g.nnz)
        rp = np.ctypeslib.as_array(g.row_ptr, shape=(n + 1,)).copy()
        cl = np.ctypeslib.as_array(g.col, shape=(max(nnz, 1),))[:nnz].copy()
    finally:
        _lib().nwgen_free(C.byref(g))
    return CSR(rp, cl)


def rmat(scale: int, edge_factor: float = 16, seed: int = 42, abc=RMAT_ABC, nthreads: int = 0) -> CSR:
    """Symmetrised, deduplicated RMAT graph with 2^scale vertices."""
    g = _Csr()
    rc = _lib().nwgen_rmat(int(scale), float(edge_factor), abc[0], abc[1], abc[2], int(seed), int(nthreads), C.byref(g))
    return _take(rc, g, "nwgen_rmat")


def grid(n_target: int) -> CSR:
    """floor(sqrt(n))^2-vertex 4-neighbour grid."""
    g = _Csr()
    return _take(_lib().nwgen_grid(int(n_target), C.byref(g)), g, "nwgen_grid")


def from_edges(src, dst, n: int, symmetrize: bool = False) -> CSR:
    """adjacency<1> (row = destination) from a directed edge list; rows sorted, duplicates dropped."""
    s = np.ascontiguousarray(src, np.uint32)
    d = np.ascontiguousarray(dst, np.uint32)
    g = _Csr()
    rc = _lib().nwgen_from_edges(s.ctypes.data_as(C.POINTER(C.c_uint32)), d.ctypes.data_as(C.POINTER(C.c_uint32)),
                                 len(s), int(n), int(bool(symmetrize)), 0, C.byref(g))
    return _take(rc, g, "nwgen_from_edges")


def random_sources(deg: np.ndarray, k: int, seed: int = 7) -> np.ndarray:
    """k vertices drawn uniformly among those with out-degree >= 1
    (as bench/gapbs/common.hpp:123-137 draws its sources)."""
    rng = np.random.default_rng(seed)
    cand = np.nonzero(deg > 0)[0]
    if len(cand) == 0:
        raise ValueError("graph has no vertex with out-degree >= 1")
    return cand[rng.integers(0, len(cand), size=k)].astype(np.uint32)


def edge_weights(nnz: int, seed: int = 1234, lo: float = 0.1, hi: float = 1.0) -> np.ndarray:
    """FP32 edge weights uniform in (lo, hi), one per CSR entry."""
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=nnz).astype(np.float32)
