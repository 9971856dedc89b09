"""Graph construction on the device (``nwgpu_csr_from_edges``,
``nwgpu_rmat_edges``, ``nwgpu_grid_edges``).

The reference builds its CSR on the host: an edge list, optionally
``remove_self_loops`` and ``uniq`` (include/nwgraph/build.hpp:394-410), then
``fill_directed`` / ``fill_undirected`` (:209-272) into ``adjacency<idx>``.
:func:`csr_from_edges` does the same steps on the GPU as radix sorts of packed
keys. :func:`rmat` and :func:`grid` generate their edge lists on the device
with the host builder's samples (``graphs.rmat`` / ``graphs.grid``) and build
them there, so they return the same CSR many times faster.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .graphs import CSR, RMAT_ABC

DEVICE_PTRS = 0x1
BY_SOURCE = 0x2
UNDIRECTED = 0x4
REMOVE_SELF_LOOPS = 0x8
UNIQUE = 0x10
UNIQUE_ENTRIES = 0x20
# the host builder's clean-up of generated graphs (graphgen.cpp): a simple symmetric graph
SIMPLE_UNDIRECTED = UNDIRECTED | REMOVE_SELF_LOOPS | UNIQUE_ENTRIES


def csr_from_edges(src, dst, n: int, flags: int = 0):
    """CSR of the edge list ``src[e] -> dst[e]`` over ``n`` vertices.

    Host arrays in, ``(CSR, degrees)`` out as numpy; CUDA tensors in, device
    tensors ``(row_ptr, col, degrees)`` out. ``flags``: BY_SOURCE,
    UNDIRECTED, REMOVE_SELF_LOOPS, UNIQUE, UNIQUE_ENTRIES (include/nwgpu.h).
    """
    m = len(src)
    if hasattr(src, "is_cuda") and src.is_cuda:
        import torch
        total = 2 * m if flags & UNDIRECTED else m
        rp = torch.empty(n + 1, dtype=torch.int32, device=src.device)
        cl = torch.empty(max(total, 1), dtype=torch.int32, device=src.device)
        deg = torch.empty(n, dtype=torch.int32, device=src.device)
        nnz = C.c_uint64()
        stream = torch.cuda.current_stream(src.device).cuda_stream
        N.check(N.lib().nwgpu_csr_from_edges(src.data_ptr(), dst.data_ptr(), m, n, flags | DEVICE_PTRS, rp.data_ptr(),
                                             cl.data_ptr(), cl.numel(), C.byref(nnz), deg.data_ptr(), stream))
        return rp, cl[: nnz.value], deg
    s = np.ascontiguousarray(src, np.uint32)
    d = np.ascontiguousarray(dst, np.uint32)
    total = 2 * m if flags & UNDIRECTED else m
    rp = np.empty(n + 1, np.uint32)
    cl = np.empty(max(total, 1), np.uint32)
    deg = np.empty(n, np.uint32)
    nnz = C.c_uint64()
    N.check(N.lib().nwgpu_csr_from_edges(s.ctypes.data, d.ctypes.data, m, n, flags & ~DEVICE_PTRS, rp.ctypes.data,
                                         cl.ctypes.data, cl.size, C.byref(nnz), deg.ctypes.data, None))
    return CSR(rp, cl[: nnz.value].copy()), deg


def _edges(m, device):
    import torch
    return (torch.empty(max(m, 1), dtype=torch.int32, device=device),
            torch.empty(max(m, 1), dtype=torch.int32, device=device))


def rmat_edges(scale: int, m: int, seed: int = 42, abc=RMAT_ABC, n: int = 0, device="cuda"):
    """m seeded RMAT samples as two int32 device tensors (ids modulo n when 0 < n < 2^scale)."""
    import torch
    src, dst = _edges(m, device)
    stream = torch.cuda.current_stream(src.device).cuda_stream
    N.check(N.lib().nwgpu_rmat_edges(int(scale), int(m), abc[0], abc[1], abc[2], int(seed), int(n), src.data_ptr(),
                                     dst.data_ptr(), stream))
    return src[:m], dst[:m]


def grid_edges(side: int, device="cuda"):
    """The side x side 4-neighbour grid's 2 side (side - 1) edges on the device."""
    import torch
    m = 2 * side * (side - 1)
    src, dst = _edges(m, device)
    stream = torch.cuda.current_stream(src.device).cuda_stream
    N.check(N.lib().nwgpu_grid_edges(int(side), src.data_ptr(), dst.data_ptr(), stream))
    return src[:m], dst[:m]


def rmat(scale: int, edge_factor: float = 16, seed: int = 42, abc=RMAT_ABC, device_out: bool = False):
    """``graphs.rmat`` built on the device: the same symmetrised simple graph.
    Returns a host CSR, or device tensors ``(row_ptr, col, degrees)``."""
    m = int(np.floor(edge_factor * (1 << scale) + 0.5))  # llround, as the host builder
    src, dst = rmat_edges(scale, m, seed, abc)
    rp, cl, deg = csr_from_edges(src, dst, 1 << scale, SIMPLE_UNDIRECTED)
    del src, dst
    if device_out:
        return rp, cl, deg
    return CSR(rp.cpu().numpy().view(np.uint32), cl.cpu().numpy().view(np.uint32))


def grid(n_target: int, device_out: bool = False):
    """``graphs.grid`` built on the device."""
    side = max(1, int(np.floor(np.sqrt(n_target))))
    while (side + 1) * (side + 1) <= n_target:
        side += 1
    while side * side > n_target:
        side -= 1
    side = max(side, 1)
    src, dst = grid_edges(side)
    rp, cl, deg = csr_from_edges(src, dst, side * side, UNDIRECTED)
    if device_out:
        return rp, cl, deg
    return CSR(rp.cpu().numpy().view(np.uint32), cl.cpu().numpy().view(np.uint32))


def ragged_sizes(num_graphs: int, max_n: float = 1e6, seed: int = 11):
    """Vertex counts (log-uniform in [1e3, max_n]) and RMAT edge factors
    (U{8..32}) of the ragged configuration's graphs."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(1e3), np.log(max_n), num_graphs)).astype(np.int64)
    return ns, rng.integers(8, 33, num_graphs)


def ragged_graphs(num_graphs: int, max_n: float = 1e6, seed: int = 11, graphs=None):
    """The ragged configuration, built on the GPU: n_g log-uniform in
    [1e3, max_n] (seed 11); even graph ids symmetrised RMAT (edge factor
    U{8..32}, scale ceil(log2 n_g), ids taken modulo n_g, self-loops and
    repeats dropped), odd ids floor(sqrt(n_g))^2 4-neighbour grids. Returns the
    device CSRs [(row_ptr, col)] and degrees of the graphs ``graphs`` (an
    iterable of ids; all of them by default)."""
    import math
    ns, efs = ragged_sizes(num_graphs, max_n, seed)
    parts, degs = [], []
    for g in (range(num_graphs) if graphs is None else graphs):
        n = int(ns[g])
        if g % 2 == 0:
            src, dst = rmat_edges(max(1, math.ceil(math.log2(n))), int(efs[g]) * n, seed=seed + g, n=n)
            rp, cl, dg = csr_from_edges(src, dst, n, SIMPLE_UNDIRECTED)
            del src, dst
        else:
            rp, cl, dg = grid(n, device_out=True)
        parts.append((rp, cl))
        degs.append(dg)
    return parts, degs


def batch_from_device_csrs(parts, degrees=None):
    """A :class:`GraphBatch` from device-built graphs ``[(row_ptr, col), ...]``
    (int32 CUDA tensors, local ids), concatenated on the device in order.
    Releases ``parts`` as it goes (the list is emptied). With ``degrees`` (a
    list of per-graph degree tensors, emptied likewise) also returns their
    concatenation."""
    import torch
    from .pagerank import GraphBatch
    dev = parts[0][0].device
    ns = np.array([int(rp.numel()) - 1 for rp, _ in parts], np.uint64)
    ms = np.array([int(cl.numel()) for _, cl in parts], np.uint64)
    vo = np.zeros(len(parts) + 1, np.uint64)
    eo = np.zeros(len(parts) + 1, np.uint64)
    vo[1:] = np.cumsum(ns)
    eo[1:] = np.cumsum(ms)
    rp_all = torch.empty(int(vo[-1]) + len(parts), dtype=torch.int32, device=dev)
    cl_all = torch.empty(max(int(eo[-1]), 1), dtype=torch.int32, device=dev)
    deg_all = torch.empty(max(int(vo[-1]), 1), dtype=torch.int32, device=dev) if degrees is not None else None
    for g in range(len(parts)):
        rp, cl = parts[g]
        p0 = int(vo[g]) + g
        rp_all[p0:p0 + rp.numel()] = rp
        cl_all[int(eo[g]):int(eo[g + 1])] = cl
        parts[g] = None
        if degrees is not None:
            deg_all[int(vo[g]):int(vo[g + 1])] = degrees[g]
            degrees[g] = None
    parts.clear()
    if degrees is not None:
        degrees.clear()
    torch.cuda.empty_cache()  # the freed parts, for the batch's own copy
    b = GraphBatch(vo, eo, rp_all, cl_all[: int(eo[-1])])
    del rp_all, cl_all
    return (b, deg_all[: int(vo[-1])]) if degrees is not None else b


def read_edges(path: str, values: bool = False, nthreads: int = 0):
    """The edge list of a graph file (Matrix Market or NW binary edge list),
    as the reference driver's load_graph reads it: ``(src, dst, n)`` uint32
    numpy arrays, plus the values when ``values``. Host code (no GPU)."""
    info = N.EdgeFile()
    N.check(N.lib().nwgpu_edge_file_probe(path.encode(), C.byref(info)))
    cap = int(info.max_edges)
    src = np.empty(max(cap, 1), np.uint32)
    dst = np.empty(max(cap, 1), np.uint32)
    val = np.empty(max(cap, 1), np.float32) if values else None
    m = C.c_uint64()
    N.check(N.lib().nwgpu_edge_file_read(path.encode(), src.ctypes.data, dst.ctypes.data,
                                         val.ctypes.data if values else None, cap, C.byref(m), int(nthreads)))
    k = m.value
    out = (src[:k].copy(), dst[:k].copy(), int(info.n))
    return out + (val[:k].copy(),) if values else out


def write_nw_edges(path: str, src, dst, n: int, directed: bool = True):
    """Write an NW binary edge list (what edge_list::deserialize reads)."""
    s = np.ascontiguousarray(src, np.uint32)
    d = np.ascontiguousarray(dst, np.uint32)
    N.check(N.lib().nwgpu_edge_file_write_nw(path.encode(), s.ctypes.data, d.ctypes.data, len(s), int(n),
                                             1 if directed else 0))


def read_adjacency(path: str):
    """A serialized NWGraph adjacency file as its CSR (host arrays)."""
    n, nnz = C.c_uint64(), C.c_uint64()
    N.check(N.lib().nwgpu_adjacency_file_read(path.encode(), None, None, None, 0, 0, C.byref(n), C.byref(nnz)))
    rp = np.empty(n.value + 1, np.uint32)
    cl = np.empty(max(nnz.value, 1), np.uint32)
    N.check(N.lib().nwgpu_adjacency_file_read(path.encode(), rp.ctypes.data, cl.ctypes.data, None, n.value, nnz.value,
                                              C.byref(n), C.byref(nnz)))
    return CSR(rp, cl[: nnz.value].copy())


def load_graph(path: str, nthreads: int = 0):
    """The reference driver's graph input (bench/gapbs/common.hpp:83-100 then
    build_adjacency<1>): the file's edge list built into adjacency<1> (row v
    lists the sources of the edges into v, rows sorted) on the GPU. Returns
    ``(CSR, degrees)`` on the host; degrees are build_degrees' out-degrees."""
    info = N.EdgeFile()
    N.check(N.lib().nwgpu_edge_file_probe(path.encode(), C.byref(info)))
    if info.format == N.FILE_NW_ADJACENCY:  # already a CSR
        g = read_adjacency(path)
        return g, np.bincount(g.col, minlength=g.n).astype(np.uint32)
    src, dst, n = read_edges(path, nthreads=nthreads)
    return csr_from_edges(src, dst, n, 0)
