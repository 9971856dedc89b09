"""Python mirror of ``nw::graph::page_rank`` on the B200 engine.

The reference call (include/nwgraph/algorithms/page_rank.hpp:89-91)::

    page_rank(graph, degrees, page_rank, damping_factor, threshold, max_iters, num_threads)

keeps its parameter list here: ``graph`` is a compressed adjacency<1>
(``row_ptr``/``col`` arrays, or any object exposing NWGraph's public
``indices_`` / ``to_be_indexed_`` members), ``degrees`` the out-degrees,
``page_rank`` a pre-sized float32 buffer that is fully overwritten, and
``num_threads`` is accepted and ignored exactly as in the reference (where it
is unused; parallelism comes from the device). Semantics are those of
``page_rank_v10`` (experimental/algorithms/page_rank.hpp:377-432): Jacobi
sweeps, FP32 scores, FP64 L1 error, stop after the first sweep whose error is
below ``threshold`` or after ``max_iters`` sweeps. Failures raise
:class:`NwgpuError` (the C++ layer throws ``std::runtime_error``); there is
no CPU fallback.

Arrays may be host numpy arrays or CUDA tensors (``torch``), which are
passed to the engine as device pointers without a host round trip.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from ._native import NwgpuError


def _is_cuda_tensor(x) -> bool:
    return hasattr(x, "is_cuda") and bool(getattr(x, "is_cuda"))


def _ptr(x, dtype):
    """(address, on_device, keepalive) for a numpy array or a torch tensor."""
    if x is None:
        return None, False, None
    if _is_cuda_tensor(x):
        import torch
        want = {np.uint32: (torch.int32, torch.uint32), np.float32: (torch.float32,), np.float64: (torch.float64,)}
        if x.dtype not in want[dtype]:
            raise TypeError(f"tensor dtype {x.dtype} does not match {np.dtype(dtype).name}")
        if not x.is_contiguous():
            raise ValueError("device tensors must be contiguous")
        return x.data_ptr(), True, x
    if hasattr(x, "is_cuda"):  # CPU torch tensor
        x = x.numpy()
    a = np.ascontiguousarray(x, dtype=dtype)
    return a.ctypes.data, False, a


def _csr_arrays(graph):
    """row_ptr, col of an adjacency<1>-like object."""
    if hasattr(graph, "indices_") and hasattr(graph, "to_be_indexed_"):
        tbi = graph.to_be_indexed_
        return graph.indices_, (tbi[0] if isinstance(tbi, (tuple, list)) else tbi)
    return graph.row_ptr, graph.col


@dataclass
class PageRankStats:
    iterations: int
    final_error: float
    converged: bool
    device_ms: float
    ms_per_iter: float
    bytes_per_iter: float
    gteps: float
    errors: np.ndarray | None = None


@dataclass
class PprBatchStats:
    iterations: int
    all_converged: bool
    device_ms: float
    ms_per_iter: float
    bytes_per_iter: float
    col_iterations: np.ndarray
    col_errors: np.ndarray
    col_converged: np.ndarray


class Graph:
    """A CSR resident in HBM (one ``nwgpu_graph`` handle).

    Upload once, solve many times: the reference re-reads ``graph.indices_`` /
    ``to_be_indexed_`` on every call (page_rank.hpp:129); here the arrays are
    copied, validated and tiled on the device at construction.
    """

    def __init__(self, row_ptr, col, weights=None, n=None, nnz=None, relabel=True, autotune=False):
        rp, rp_dev, self._k0 = _ptr(row_ptr, np.uint32)
        cl, cl_dev, self._k1 = _ptr(col, np.uint32)
        w, w_dev, self._k2 = _ptr(weights, np.float32)
        if len({rp_dev, cl_dev} | ({w_dev} if weights is not None else set())) != 1:
            raise ValueError("row_ptr, col and weights must all be on the host or all on the device")
        self.n = int(n if n is not None else len(row_ptr) - 1)
        self.nnz = int(nnz if nnz is not None else len(col))
        flags = ((N.GRAPH_DEVICE_PTRS if rp_dev else 0) | (0 if relabel else N.GRAPH_NO_RELABEL)
                 | (N.GRAPH_AUTOTUNE if autotune else 0))
        h = C.c_void_p()
        N.check(N.lib().nwgpu_graph_create(rp, cl, w, self.n, self.nnz, flags, C.byref(h)))
        self._h = h
        self._k0 = self._k1 = self._k2 = None

    @classmethod
    def from_adjacency(cls, graph, weights=None):
        rp, cl = _csr_arrays(graph)
        return cls(rp, cl, weights)

    @property
    def handle(self):
        if self._h is None:
            raise ValueError("graph was released")
        return self._h

    def info(self) -> dict:
        gi = N.GraphInfo()
        N.check(N.lib().nwgpu_graph_get_info(self.handle, C.byref(gi)))
        return {f: getattr(gi, f) for f, _ in gi._fields_}

    def release(self):
        if getattr(self, "_h", None) is not None:
            N.lib().nwgpu_graph_destroy(self._h)
            self._h = None

    close = release

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.release()

    def abort(self):
        N.check(N.lib().nwgpu_abort(self.handle))

    # ------------------------------------------------------------------
    def _vectors(self, degrees, out, n_out):
        if len(degrees) != self.n:
            raise ValueError(f"degrees must have {self.n} entries")
        dp, d_dev, keep = _ptr(degrees, np.uint32)
        out_dev = _is_cuda_tensor(out)
        if d_dev != out_dev:
            raise ValueError("degrees and outputs must both be host arrays or both device tensors")
        if out_dev:
            if str(out.dtype) != "torch.float32" or not out.is_contiguous() or out.numel() != n_out:
                raise TypeError(f"output must be a contiguous float32 tensor of {n_out} entries")
            op = out.data_ptr()
        else:
            if not (isinstance(out, np.ndarray) and out.dtype == np.float32 and out.flags.c_contiguous
                    and out.size == n_out):
                raise TypeError(f"output must be a contiguous float32 numpy array of {n_out} entries (filled in place)")
            op = out.ctypes.data
        return dp, op, out_dev, keep

    def _options(self, launch, device, stream):
        opt = N.PrOptions(size=C.sizeof(N.PrOptions), mode=N.MODE_PARITY,
                          launch=N.LAUNCH_STREAM if launch == "stream" else N.LAUNCH_GRAPH,
                          device_ptrs=1 if device else 0)
        if stream is not None:
            opt.stream = int(getattr(stream, "cuda_stream", stream))
        return opt

    def page_rank_residual(self, degrees, out, damping_factor=0.85, threshold=1e-4, max_iters=20, launch="graph",
                           record_errors=False, stream=None) -> PageRankStats:
        """Residual-push PageRank (page_rank_v13; nwgpu_pr_residual_run). Ranks are not normalised."""
        dp, op, dev, keep = self._vectors(degrees, out, self.n)
        opt = self._options(launch, dev, stream)
        st = N.PrStats()
        errs = None
        if record_errors:
            cap = int(min(max(int(max_iters), 1), 4096))
            errs = np.zeros(cap, np.float64)
            st.errors = errs.ctypes.data_as(C.POINTER(C.c_double))
            st.errors_cap = cap
        N.check(N.lib().nwgpu_pr_residual_run(self.handle, dp, op, C.c_float(damping_factor), C.c_float(threshold),
                                              int(max_iters), C.byref(opt), C.byref(st)))
        del keep
        return PageRankStats(int(st.iterations), float(st.final_error), bool(st.converged), float(st.device_ms),
                             float(st.ms_per_iter), float(st.bytes_per_iter), float(st.gteps),
                             None if errs is None else errs[: min(int(st.iterations), len(errs))])

    def ppr(self, degrees, seed, out, damping_factor=0.85, threshold=1e-6, max_iters=100, launch="graph",
            record_errors=False, stream=None) -> PageRankStats:
        """Personalised PageRank with a one-hot teleport at ``seed`` (nwgpu_ppr_run)."""
        dp, op, dev, keep = self._vectors(degrees, out, self.n)
        opt = self._options(launch, dev, stream)
        st = N.PrStats()
        errs = None
        if record_errors:
            cap = int(min(max(int(max_iters), 1), 4096))
            errs = np.zeros(cap, np.float64)
            st.errors = errs.ctypes.data_as(C.POINTER(C.c_double))
            st.errors_cap = cap
        N.check(N.lib().nwgpu_ppr_run(self.handle, dp, int(seed), op, C.c_float(damping_factor), C.c_float(threshold),
                                      int(max_iters), C.byref(opt), C.byref(st)))
        del keep
        return PageRankStats(int(st.iterations), float(st.final_error), bool(st.converged), float(st.device_ms),
                             float(st.ms_per_iter), float(st.bytes_per_iter), float(st.gteps),
                             None if errs is None else errs[: min(int(st.iterations), len(errs))])

    def weighted_page_rank_batched(self, teleports, out, damping_factor=0.85, threshold=1e-6, max_iters=100,
                                   launch="graph", stream=None) -> PprBatchStats:
        """k weighted personalised vectors at once (nwgpu_wppr_batched); ``teleports`` and ``out`` are n x k
        row-major float32 (host arrays or CUDA tensors)."""
        if len(teleports.shape) != 2 or tuple(out.shape) != tuple(teleports.shape):
            raise ValueError("teleports and out must be n x k matrices")
        k = int(teleports.shape[1])
        (tp, op), dev, keep = self._f32_vectors([teleports.reshape(-1), out.reshape(-1)], [self.n * k, self.n * k])
        opt = self._options(launch, dev, stream)
        ci = np.zeros(k, np.uint32)
        ce = np.zeros(k, np.float64)
        cc = np.zeros(k, np.int32)
        st = N.PprStats()
        st.col_iterations = ci.ctypes.data_as(C.POINTER(C.c_uint32))
        st.col_errors = ce.ctypes.data_as(C.POINTER(C.c_double))
        st.col_converged = cc.ctypes.data_as(C.POINTER(C.c_int32))
        N.check(N.lib().nwgpu_wppr_batched(self.handle, tp, k, op, C.c_float(damping_factor), C.c_float(threshold),
                                           int(max_iters), C.byref(opt), C.byref(st)))
        del keep
        return PprBatchStats(int(st.iterations), bool(st.all_converged), float(st.device_ms), float(st.ms_per_iter),
                             float(st.bytes_per_iter), ci, ce, cc.astype(bool))

    def ppr_batched_teleports(self, degrees, teleports, out, damping_factor=0.85, threshold=1e-6, max_iters=100,
                              launch="graph", stream=None) -> PprBatchStats:
        """k personalised vectors with teleport vectors on an unweighted graph (nwgpu_ppr_batched_teleports);
        ``teleports`` and ``out`` are n x k row-major float32, host arrays or CUDA tensors like ``degrees``."""
        if len(teleports.shape) != 2 or tuple(out.shape) != tuple(teleports.shape):
            raise ValueError("teleports and out must be n x k matrices")
        if len(degrees) != self.n:
            raise ValueError(f"degrees must have {self.n} entries")
        k = int(teleports.shape[1])
        (tp, op), dev, keep = self._f32_vectors([teleports.reshape(-1), out.reshape(-1)], [self.n * k, self.n * k])
        dp, d_dev, keep_d = _ptr(degrees, np.uint32)
        if self.n and d_dev != dev:
            raise ValueError("degrees, teleports and out must all be host arrays or all device tensors")
        opt = self._options(launch, dev, stream)
        ci = np.zeros(k, np.uint32)
        ce = np.zeros(k, np.float64)
        cc = np.zeros(k, np.int32)
        st = N.PprStats()
        st.col_iterations = ci.ctypes.data_as(C.POINTER(C.c_uint32))
        st.col_errors = ce.ctypes.data_as(C.POINTER(C.c_double))
        st.col_converged = cc.ctypes.data_as(C.POINTER(C.c_int32))
        N.check(N.lib().nwgpu_ppr_batched_teleports(self.handle, dp, tp, k, op, C.c_float(damping_factor),
                                                    C.c_float(threshold), int(max_iters), C.byref(opt), C.byref(st)))
        del keep, keep_d
        return PprBatchStats(int(st.iterations), bool(st.all_converged), float(st.device_ms), float(st.ms_per_iter),
                             float(st.bytes_per_iter), ci, ce, cc.astype(bool))

    def ppr_batched(self, degrees, seeds, out, damping_factor=0.85, threshold=1e-6, max_iters=100, launch="graph",
                    stream=None) -> PprBatchStats:
        """k personalised vectors at once (nwgpu_ppr_batched); ``out`` is n x k row-major float32."""
        seeds_h = np.ascontiguousarray(np.asarray(seeds.cpu() if hasattr(seeds, "cpu") else seeds), np.uint32)
        k = len(seeds_h)
        dp, op, dev, keep = self._vectors(degrees, out, self.n * k)
        if dev:
            import torch
            seeds_arg = torch.from_numpy(seeds_h.view(np.int32)).to(out.device)
            sp = seeds_arg.data_ptr()
        else:
            seeds_arg = seeds_h
            sp = seeds_h.ctypes.data
        opt = self._options(launch, dev, stream)
        ci = np.zeros(k, np.uint32)
        ce = np.zeros(k, np.float64)
        cc = np.zeros(k, np.int32)
        st = N.PprStats()
        st.col_iterations = ci.ctypes.data_as(C.POINTER(C.c_uint32))
        st.col_errors = ce.ctypes.data_as(C.POINTER(C.c_double))
        st.col_converged = cc.ctypes.data_as(C.POINTER(C.c_int32))
        N.check(N.lib().nwgpu_ppr_batched(self.handle, dp, sp, k, op, C.c_float(damping_factor), C.c_float(threshold),
                                          int(max_iters), C.byref(opt), C.byref(st)))
        del keep, seeds_arg
        return PprBatchStats(int(st.iterations), bool(st.all_converged), float(st.device_ms), float(st.ms_per_iter),
                             float(st.bytes_per_iter), ci, ce, cc.astype(bool))

    def page_rank(self, degrees, page_rank, damping_factor=0.85, threshold=1e-4, max_iters=20,
                  launch: str = "graph", record_errors: bool = False, stream=None) -> PageRankStats:
        """Solve into ``page_rank`` (fully overwritten). Returns the stats.

        ``stream`` (a ``torch.cuda.Stream`` or raw ``cudaStream_t`` int) runs the
        solve on the caller's stream instead of the handle's own.
        """
        if len(page_rank) != self.n or len(degrees) != self.n:
            raise ValueError(f"degrees/page_rank must have {self.n} entries")
        dp, d_dev, keep_d = _ptr(degrees, np.uint32)
        out_dev = _is_cuda_tensor(page_rank)
        if d_dev != out_dev:
            raise ValueError("degrees and page_rank must both be host arrays or both device tensors")
        if out_dev:
            if page_rank.dtype.__str__() != "torch.float32" or not page_rank.is_contiguous():
                raise TypeError("page_rank must be a contiguous float32 tensor")
            rp = page_rank.data_ptr()
            host_out = None
        else:
            if not (isinstance(page_rank, np.ndarray) and page_rank.dtype == np.float32
                    and page_rank.flags.c_contiguous):
                raise TypeError("page_rank must be a contiguous float32 numpy array (filled in place)")
            host_out = page_rank
            rp = host_out.ctypes.data
        opt = N.PrOptions(size=C.sizeof(N.PrOptions), mode=N.MODE_PARITY,
                          launch=N.LAUNCH_STREAM if launch == "stream" else N.LAUNCH_GRAPH,
                          device_ptrs=1 if out_dev else 0)
        if stream is not None:
            opt.stream = int(getattr(stream, "cuda_stream", stream))
        st = N.PrStats()
        errs = None
        if record_errors:
            cap = int(min(max(int(max_iters), 1), 4096))
            errs = np.zeros(cap, np.float64)
            st.errors = errs.ctypes.data_as(C.POINTER(C.c_double))
            st.errors_cap = cap
        N.check(N.lib().nwgpu_pr_run(self.handle, dp, rp, C.c_float(damping_factor), C.c_float(threshold),
                                     int(max_iters), C.byref(opt), C.byref(st)))
        del keep_d
        return PageRankStats(int(st.iterations), float(st.final_error), bool(st.converged), float(st.device_ms),
                             float(st.ms_per_iter), float(st.bytes_per_iter), float(st.gteps),
                             None if errs is None else errs[: min(int(st.iterations), len(errs))])


    # ------------------------------------------------------------------
    def _f32_vectors(self, arrays, sizes):
        """Addresses of float32 vectors that are all host arrays or all CUDA
        tensors (None allowed); outputs are filled in place."""
        dev = {_is_cuda_tensor(x) for x in arrays if x is not None}
        if len(dev) > 1:
            raise ValueError("vectors must all be host arrays or all device tensors")
        on_dev = dev.pop() if dev else False
        ptrs, keep = [], []
        for x, size in zip(arrays, sizes):
            if x is None:
                ptrs.append(None)
                continue
            if len(x) != size:
                raise ValueError(f"expected {size} entries, got {len(x)}")
            if on_dev:
                if str(x.dtype) != "torch.float32" or not x.is_contiguous():
                    raise TypeError("device vectors must be contiguous float32 tensors")
                ptrs.append(x.data_ptr())
            else:
                if not (isinstance(x, np.ndarray) and x.dtype == np.float32 and x.flags.c_contiguous):
                    raise TypeError("host vectors must be contiguous float32 numpy arrays")
                ptrs.append(x.ctypes.data)
            keep.append(x)
        return ptrs, on_dev, keep

    @staticmethod
    def _stats(st, errs):
        return PageRankStats(int(st.iterations), float(st.final_error), bool(st.converged), float(st.device_ms),
                             float(st.ms_per_iter), float(st.bytes_per_iter), float(st.gteps),
                             None if errs is None else errs[: min(int(st.iterations), len(errs))])

    @staticmethod
    def _error_buffer(st, record, max_iters):
        if not record:
            return None
        cap = int(min(max(int(max_iters), 1), 4096))
        errs = np.zeros(cap, np.float64)
        st.errors = errs.ctypes.data_as(C.POINTER(C.c_double))
        st.errors_cap = cap
        return errs

    def weighted_page_rank(self, teleport, out, damping_factor=0.85, threshold=1e-6, max_iters=100, launch="graph",
                           record_errors=False, stream=None) -> PageRankStats:
        """Weighted PageRank with a teleport distribution (nwgpu_wpr_run):
        r = (1-d) t + d W^T D_s^-1 r over the edge weights given at creation.
        ``teleport`` has n entries (None: uniform 1/n); ``out`` is filled in place."""
        (tp, op), dev, keep = self._f32_vectors([teleport, out], [self.n, self.n])
        opt = self._options(launch, dev, stream)
        st = N.PrStats()
        errs = self._error_buffer(st, record_errors, max_iters)
        N.check(N.lib().nwgpu_wpr_run(self.handle, tp, op, C.c_float(damping_factor), C.c_float(threshold),
                                      int(max_iters), C.byref(opt), C.byref(st)))
        del keep
        return self._stats(st, errs)

    def spmv(self, x, y, stream=None):
        """y = A x over the rows (nwgpu_spmv): y[i] = sum_k weights[k] * x[col[k]] for row i's entries."""
        (xp, yp), dev, keep = self._f32_vectors([x, y], [self.n, self.n])
        opt = self._options("stream", dev, stream)
        N.check(N.lib().nwgpu_spmv(self.handle, xp, yp, C.byref(opt)))
        del keep

    def page_rank_vjp(self, ranks, dL_dr, dL_dw=None, dL_dt=None, damping_factor=0.85, threshold=1e-7,
                      max_iters=1000, launch="graph", record_errors=False, stream=None) -> PageRankStats:
        """Gradients of L = dL_dr . r at the weighted fixed point ``ranks``
        (nwgpu_pr_vjp): dL/dw (nnz, input entry order) and dL/dt (n), each
        filled in place when given. Returns the adjoint solve's stats."""
        (rp, cp, wp, tp), dev, keep = self._f32_vectors([ranks, dL_dr, dL_dw, dL_dt],
                                                        [self.n, self.n, self.nnz, self.n])
        opt = self._options(launch, dev, stream)
        st = N.PrStats()
        errs = self._error_buffer(st, record_errors, max_iters)
        N.check(N.lib().nwgpu_pr_vjp(self.handle, rp, cp, wp, tp, C.c_float(damping_factor), C.c_float(threshold),
                                     int(max_iters), C.byref(opt), C.byref(st)))
        del keep
        return self._stats(st, errs)


@dataclass
class RaggedStats:
    sweeps: int
    converged_graphs: int
    device_ms: float
    entries_swept: float
    gteps: float
    graph_iterations: np.ndarray
    graph_errors: np.ndarray
    graph_converged: np.ndarray


class GraphBatch:
    """Many independent graphs resident in HBM (one ``nwgpu_batch`` handle),
    solved together by :meth:`page_rank` with per-graph convergence.

    Graph ``g`` is a CSR with local ids: ``row_ptr[vertex_offsets[g] + g :
    vertex_offsets[g + 1] + g + 1]`` are its row pointers (first 0) and
    ``col[entry_offsets[g] : entry_offsets[g + 1]]`` its column ids.
    Per-vertex arrays (degrees, ranks) are concatenated in graph order, graph
    ``g``'s at ``vertex_offsets[g]``. No counterpart in the reference: each
    graph gets what ``page_rank`` (page_rank.hpp:92-147) gives for it alone.
    Graphs of at least 2^22 entries (NWGPU_RAGGED_SOLO_ENTRIES, read when the
    batch is created) are solved by single-graph handles beside the batch.
    """

    def __init__(self, vertex_offsets, entry_offsets, row_ptr, col):
        self.vertex_offsets = np.ascontiguousarray(vertex_offsets, np.uint64)
        self.entry_offsets = np.ascontiguousarray(entry_offsets, np.uint64)
        if self.vertex_offsets.shape != self.entry_offsets.shape or self.vertex_offsets.size < 2:
            raise ValueError("vertex_offsets and entry_offsets need num_graphs + 1 entries each")
        self.num_graphs = self.vertex_offsets.size - 1
        self.n = int(self.vertex_offsets[-1])
        self.nnz = int(self.entry_offsets[-1])
        rp, rp_dev, k0 = _ptr(row_ptr, np.uint32)
        cl, cl_dev, k1 = _ptr(col, np.uint32)
        if self.nnz and rp_dev != cl_dev:
            raise ValueError("row_ptr and col must both be on the host or both on the device")
        if len(row_ptr) != self.n + self.num_graphs or len(col) != self.nnz:
            raise ValueError("row_ptr needs n + num_graphs entries and col entry_offsets[-1]")
        h = C.c_void_p()
        N.check(N.lib().nwgpu_batch_create(self.num_graphs, self.vertex_offsets.ctypes.data,
                                           self.entry_offsets.ctypes.data, rp, cl,
                                           N.GRAPH_DEVICE_PTRS if rp_dev else 0, C.byref(h)))
        self._h = h
        del k0, k1

    @classmethod
    def from_graphs(cls, graphs):
        """Batch of ``(row_ptr, col)`` pairs (or objects with ``row_ptr`` / ``col``)."""
        rps, cols = [], []
        for g in graphs:
            rp, cl = (g if isinstance(g, tuple) else _csr_arrays(g))
            rps.append(np.asarray(rp, np.uint32))
            cols.append(np.asarray(cl, np.uint32))
        vo = np.zeros(len(rps) + 1, np.uint64)
        eo = np.zeros(len(rps) + 1, np.uint64)
        vo[1:] = np.cumsum([len(r) - 1 for r in rps])
        eo[1:] = np.cumsum([len(c) for c in cols])
        return cls(vo, eo, np.concatenate(rps), np.concatenate(cols) if cols else np.zeros(0, np.uint32))

    @property
    def handle(self):
        if self._h is None:
            raise ValueError("batch was released")
        return self._h

    def release(self):
        if getattr(self, "_h", None) is not None:
            N.lib().nwgpu_batch_destroy(self._h)
            self._h = None

    close = release

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.release()

    def split(self, values):
        """Per-graph views of a concatenated per-vertex array."""
        vo = self.vertex_offsets.astype(np.int64)
        return [values[vo[g]:vo[g + 1]] for g in range(self.num_graphs)]

    def page_rank(self, degrees, page_rank, damping_factor=0.85, threshold=1e-4, max_iters=20, launch="graph",
                  stream=None) -> RaggedStats:
        """Solve every graph into ``page_rank`` (concatenated, fully overwritten)."""
        if len(degrees) != self.n or len(page_rank) != self.n:
            raise ValueError(f"degrees/page_rank must have {self.n} entries")
        dp, d_dev, keep = _ptr(degrees, np.uint32)
        out_dev = _is_cuda_tensor(page_rank)
        if self.n and d_dev != out_dev:
            raise ValueError("degrees and page_rank must both be host arrays or both device tensors")
        if out_dev:
            if str(page_rank.dtype) != "torch.float32" or not page_rank.is_contiguous():
                raise TypeError("page_rank must be a contiguous float32 tensor")
            op = page_rank.data_ptr()
        else:
            if not (isinstance(page_rank, np.ndarray) and page_rank.dtype == np.float32
                    and page_rank.flags.c_contiguous):
                raise TypeError("page_rank must be a contiguous float32 numpy array (filled in place)")
            op = page_rank.ctypes.data
        opt = N.PrOptions(size=C.sizeof(N.PrOptions), mode=N.MODE_PARITY,
                          launch=N.LAUNCH_STREAM if launch == "stream" else N.LAUNCH_GRAPH,
                          device_ptrs=1 if out_dev else 0)
        if stream is not None:
            opt.stream = int(getattr(stream, "cuda_stream", stream))
        G = self.num_graphs
        gi = np.zeros(G, np.uint32)
        ge = np.zeros(G, np.float64)
        gc = np.zeros(G, np.int32)
        st = N.BatchStats()
        st.graph_iterations = gi.ctypes.data_as(C.POINTER(C.c_uint32))
        st.graph_errors = ge.ctypes.data_as(C.POINTER(C.c_double))
        st.graph_converged = gc.ctypes.data_as(C.POINTER(C.c_int32))
        N.check(N.lib().nwgpu_pr_ragged(self.handle, dp, op, C.c_float(damping_factor), C.c_float(threshold),
                                        int(max_iters), C.byref(opt), C.byref(st)))
        del keep
        return RaggedStats(int(st.sweeps), int(st.converged_graphs), float(st.device_ms), float(st.entries_swept),
                           float(st.gteps), gi, ge, gc.astype(bool))


def page_rank(graph, degrees, page_rank, damping_factor=0.85, threshold=1e-4, max_iters=20, num_threads=None):
    """Drop-in for ``nw::graph::page_rank`` (page_rank.hpp:89-148).

    ``graph`` may be a resident :class:`Graph` (warm call) or a CSR / adjacency
    object (uploaded for this call and released after). ``num_threads`` is
    unused, as in the reference. Returns None, like the reference; use
    :meth:`Graph.page_rank` for statistics.
    """
    del num_threads
    if isinstance(graph, Graph):
        graph.page_rank(degrees, page_rank, damping_factor, threshold, max_iters)
        return None
    with Graph.from_adjacency(graph) as g:
        g.page_rank(degrees, page_rank, damping_factor, threshold, max_iters)
    return None
