"""Row-sharded PageRank across GPUs.

The reference solves on one host (include/nwgraph/algorithms/page_rank.hpp:
89-148). Here the sweep is split by destination rows over the ranks of a
``torch.distributed`` group, one GPU each:

* every rank relabels the whole graph the same way (descending row length,
  stably, as the single-GPU engine does) and owns a contiguous range of the
  relabelled rows, chosen so that every range holds about the same number of
  rows plus entries (:func:`shard_bounds`);
* contributions live in a padded layout of ``world * stride`` floats, rank q's
  rows at ``q * stride``, so one equal-count all-gather of the ranks' slices
  (``all_gather_into_tensor`` over NCCL) rebuilds the whole vector after each
  sweep, and one all-reduce sums the ranks' FP64 L1 changes;
* every rank takes the same stopping decision from that sum: the first sweep
  whose L1 change is below ``threshold``, or ``max_iters`` (page_rank.hpp:144).

The per-rank building blocks are the engine's ``nwgpu_shard_*`` C ABI
(:class:`GpuShard`); the exchange is torch.distributed (:class:`DistExchange`),
or plain copies when one process holds every shard (:class:`LocalExchange`).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from ._native import NwgpuError


def shard_bounds(row_ptr, world: int):
    """Row ranges of ``world`` ranks over the relabelled CSR of ``row_ptr``.

    The relabelled rows are the input rows sorted by descending length; the
    ranges cut the merge path of that CSR (rows plus entries) into ``world``
    nearly equal parts. Returns ``(bounds, stride)``: ``bounds[world + 1]``
    (uint64, from 0 to n) and the slice stride (the largest range rounded up
    to a multiple of 4)."""
    rp = np.asarray(row_ptr, np.int64)
    n = len(rp) - 1
    lens = np.sort(np.diff(rp))[::-1]
    ends = np.cumsum(lens) + np.arange(1, n + 1)  # merge-path index just past each row's end item
    total = n + int(rp[-1])
    cuts = [int(np.searchsorted(ends, q * total // world, side="right")) for q in range(1, world)]
    bounds = np.maximum.accumulate(np.array([0] + cuts + [n], np.uint64))
    stride = max(4, (int(np.diff(bounds).max()) + 3) // 4 * 4)
    return bounds, stride


class GpuShard:
    """One rank's rows on this process's current GPU (``nwgpu_shard``)."""

    def __init__(self, row_ptr, col, world: int, rank: int, bounds, stride: int):
        from .pagerank import _ptr
        rp, rp_dev, k0 = _ptr(row_ptr, np.uint32)
        cl, _, k1 = _ptr(col, np.uint32)
        self.n = len(row_ptr) - 1
        self.nnz = len(col)
        self.world, self.rank, self.stride = world, rank, stride
        self._bounds = np.ascontiguousarray(bounds, np.uint64)
        h = C.c_void_p()
        N.check(N.lib().nwgpu_shard_create(rp, cl, self.n, self.nnz, world, rank, self._bounds.ctypes.data, stride,
                                           N.GRAPH_DEVICE_PTRS if rp_dev else 0, C.byref(h)))
        self._h = h
        del k0, k1

    def start(self, degrees, contrib_slice, stream):
        from .pagerank import _ptr
        dp, d_dev, keep = _ptr(degrees, np.uint32)
        N.check(N.lib().nwgpu_shard_start(self._h, dp, 1 if d_dev else 0, contrib_slice.data_ptr(), stream))
        del keep

    def sweep(self, contrib_all, contrib_slice, damping, l1, stream):
        N.check(N.lib().nwgpu_shard_sweep(self._h, contrib_all.data_ptr(), contrib_slice.data_ptr(),
                                          C.c_float(damping), l1.data_ptr(), stream))

    def decide(self, total, threshold, max_iters, state, errors, errors_cap, stream):
        N.check(N.lib().nwgpu_shard_decide(self._h, total.data_ptr(), float(threshold), int(max_iters),
                                           state.data_ptr(), errors.data_ptr() if errors is not None else None,
                                           int(errors_cap), stream))

    def rank_slice(self, out, stream):
        N.check(N.lib().nwgpu_shard_rank_slice(self._h, out.data_ptr(), stream))

    def unpermute(self, ranks_all, ranks, stream):
        N.check(N.lib().nwgpu_shard_unpermute(self._h, ranks_all.data_ptr(), ranks.data_ptr(), stream))

    def release(self):
        if getattr(self, "_h", None) is not None:
            N.lib().nwgpu_shard_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class DistExchange:
    """The exchange over a torch.distributed group (one shard per rank)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.gloo = dist.get_backend(group) == "gloo"

    def gather(self, full, slices):
        (s,) = slices
        if self.gloo:  # gloo has no all_gather_into_tensor: gather into views of `full`
            self.dist.all_gather(list(full.view(self.world, -1).unbind(0)), s, group=self.group)
        else:
            self.dist.all_gather_into_tensor(full, s, group=self.group)

    def total(self, l1):
        """The ranks' summed L1 change, left on the device (l1 holds this rank's one shard's change)."""
        self.dist.all_reduce(l1, op=self.dist.ReduceOp.SUM, group=self.group)
        return l1


class LocalExchange:
    """Every shard in this process (their kernels never wait on one another):
    slices are copied into place and the L1 changes summed in rank order."""

    def gather(self, full, slices):
        stride = slices[0].numel()
        for q, s in enumerate(slices):
            full[q * stride:(q + 1) * stride].copy_(s)

    def total(self, l1):
        """The shards' L1 changes summed in rank order, left on the device."""
        t = l1[0:1].clone()
        for j in range(1, l1.numel()):
            t += l1[j:j + 1]
        return t


@dataclass
class ShardedStats:
    iterations: int
    final_error: float
    converged: bool
    device_ms: float
    errors: list = field(default_factory=list)


def run(shards, exchange, degrees, ranks_out, damping=0.85, threshold=1e-4, max_iters=20, device=None, chunk=8):
    """The sharded solve: start, then per sweep every local shard sweeps, the
    slices are gathered, the L1 changes summed over the ranks, and every shard
    takes the stopping decision from that sum on the device (the first sweep
    whose summed change is < threshold, or max_iters; page_rank.hpp:144). The
    host does not read the change back each sweep: it queues ``chunk`` sweeps
    (each with its exchange and decision) and reads the decision state once
    per chunk. A shard that has stopped skips its later sweeps, whose
    exchanges then move unchanged slices, so every rank takes the same
    collective steps. The ranks are gathered and written to ``ranks_out`` (n
    floats, input order) on every rank. ``shards`` are this process's shards
    in rank order; ``device`` is the torch device of the buffers."""
    import torch
    dev = torch.device(device) if device is not None else (ranks_out.device if hasattr(ranks_out, "device") else None)
    stride, world = shards[0].stride, shards[0].world
    on_gpu = dev is not None and dev.type == "cuda"
    stream = torch.cuda.current_stream(dev).cuda_stream if on_gpu else None
    full = torch.zeros(world * stride, dtype=torch.float32, device=dev)
    slices = [torch.zeros(stride, dtype=torch.float32, device=dev) for _ in shards]
    l1 = torch.zeros(len(shards), dtype=torch.float64, device=dev)
    state = torch.zeros((len(shards), 4), dtype=torch.int64, device=dev)  # sweeps, stopped, converged, failed
    cap = int(min(max(int(max_iters), 1), 1 << 16))
    hist = torch.zeros(cap, dtype=torch.float64, device=dev)
    for sh, s in zip(shards, slices):
        sh.start(degrees, s, stream)
    exchange.gather(full, slices)
    if on_gpu:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
    launched, host_state = 0, [0, 0, 0, 0]
    while launched < int(max_iters):
        for _ in range(min(int(chunk), int(max_iters) - launched)):
            for j, (sh, s) in enumerate(zip(shards, slices)):
                sh.sweep(full, s, damping, l1[j:j + 1], stream)
            exchange.gather(full, slices)
            total = exchange.total(l1)
            for j, sh in enumerate(shards):
                sh.decide(total, threshold, max_iters, state[j], hist if j == 0 else None, cap, stream)
            launched += 1
        host_state = [int(x) for x in state[0].cpu()]  # one read-back per chunk
        if host_state[1]:
            break
    ms = 0.0
    if on_gpu:
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
    if host_state[3]:
        raise NwgpuError(N.ERR_CUDA, "a bounded device wait gave up on some rank")
    sweeps = host_state[0]
    errors = hist[:min(sweeps, cap)].cpu().tolist()
    for sh, s in zip(shards, slices):
        sh.rank_slice(s, stream)
    exchange.gather(full, slices)
    shards[0].unpermute(full, ranks_out, stream)
    if on_gpu:
        torch.cuda.synchronize(dev)
    return ShardedStats(sweeps, errors[-1] if errors else 0.0, bool(host_state[2]), ms, errors)


class ShardedGraph:
    """This rank's part of a row-sharded graph: the whole CSR is passed on
    every rank (host arrays or CUDA tensors), the rank keeps its rows.
    ``page_rank`` has the reference call's meaning and fills ``page_rank``
    (n floats, input order) on every rank."""

    def __init__(self, row_ptr, col, group=None):
        import torch
        self.exchange = DistExchange(group)
        self.world, self.rank = self.exchange.world, self.exchange.rank
        rp_host = row_ptr.cpu().numpy().view(np.uint32) if hasattr(row_ptr, "cpu") else np.asarray(row_ptr)
        self.bounds, self.stride = shard_bounds(rp_host, self.world)
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.shard = GpuShard(row_ptr, col, self.world, self.rank, self.bounds, self.stride)
        self.n = self.shard.n

    def page_rank(self, degrees, page_rank, damping_factor=0.85, threshold=1e-4, max_iters=20) -> ShardedStats:
        return run([self.shard], self.exchange, degrees, page_rank, damping_factor, threshold, max_iters,
                   device=self.device)

    def release(self):
        self.shard.release()


# ---- batches: personalised columns and whole graphs shard without an exchange per sweep ----

def even_bounds(count: int, world: int) -> np.ndarray:
    """``world`` contiguous ranges over ``count`` items whose sizes differ by at
    most one (the first ``count % world`` ranges hold one more). Returns
    ``bounds[world + 1]`` (int64, from 0 to ``count``)."""
    q, r = divmod(int(count), int(world))
    sizes = np.full(int(world), q, np.int64)
    sizes[:r] += 1
    return np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)


def weighted_bounds(weights, world: int) -> np.ndarray:
    """``world`` contiguous ranges of whole items with weight sums as even as
    whole items allow: cut q falls on the item boundary nearest to q / world
    of the total weight. Returns ``bounds[world + 1]`` (int64)."""
    ends = np.concatenate([[0.0], np.cumsum(np.asarray(weights, np.float64))])
    total = ends[-1]
    cuts = []
    for q in range(1, int(world)):
        t = q * total / world
        j = int(np.searchsorted(ends, t))  # ends[j - 1] < t <= ends[j]
        if j > 0 and t - ends[j - 1] <= ends[j] - t:
            j -= 1
        cuts.append(j)
    return np.maximum.accumulate(np.array([0] + cuts + [len(ends) - 1], np.int64))


def graph_bounds(vertex_offsets, entry_offsets, world: int) -> np.ndarray:
    """Graph ranges of a ragged batch over ``world`` ranks: whole graphs,
    balanced by rows plus entries (the merge-path items its sweep walks)."""
    vo = np.asarray(vertex_offsets, np.int64)
    eo = np.asarray(entry_offsets, np.int64)
    return weighted_bounds(np.diff(vo) + np.diff(eo), world)


def batch_slice(vertex_offsets, entry_offsets, row_ptr, col, lo: int, hi: int):
    """Graphs ``[lo, hi)`` of a batch in the :class:`~nwgraph_b200.GraphBatch`
    layout, as a batch of their own: ``(vertex_offsets, entry_offsets,
    row_ptr, col)`` with the offsets rebased to 0 and the arrays sliced
    (views: a graph's row pointers are local to it, so nothing is rewritten)."""
    vo = np.asarray(vertex_offsets, np.uint64)
    eo = np.asarray(entry_offsets, np.uint64)
    v0, v1, e0, e1 = int(vo[lo]), int(vo[hi]), int(eo[lo]), int(eo[hi])
    return vo[lo:hi + 1] - vo[lo], eo[lo:hi + 1] - eo[lo], row_ptr[v0 + lo:v1 + hi], col[e0:e1]


def gather_rows(local, counts, exchange):
    """The ranks' ``local`` blocks (rank q's holds ``counts[q]`` rows of one
    trailing shape) concatenated in rank order, on every rank: each block is
    padded to the largest count and one equal-size all-gather moves them."""
    import torch
    world = len(counts)
    cmax = max(int(max(counts)), 1)
    tail = tuple(local.shape[1:])
    pad = torch.zeros((cmax,) + tail, dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    full = torch.empty(world * pad.numel(), dtype=local.dtype, device=local.device)
    exchange.gather(full, [pad.reshape(-1)])
    full = full.view((world, cmax) + tail)
    return torch.cat([full[q, :int(counts[q])] for q in range(world)], 0)


def solve_columns(graph, degrees, seeds, out, bounds, rank: int, damping_factor=0.85, threshold=1e-6,
                  max_iters=100, stream=None):
    """Rank ``rank``'s share of a personalised batch: the seeds
    ``[bounds[rank], bounds[rank + 1])`` solved by ``graph.ppr_batched`` into
    ``out`` (n x that many, row-major). Returns its stats, or None for an empty
    share. A converged column is frozen and every column is summed in the same
    order whatever the other columns are, so the shares are the columns of
    one whole batch."""
    lo, hi = int(bounds[rank]), int(bounds[rank + 1])
    if hi == lo:
        return None
    kw = {} if stream is None else {"stream": stream}
    return graph.ppr_batched(degrees, seeds[lo:hi], out, damping_factor, threshold, max_iters, **kw)


@dataclass
class ShardedPprStats:
    iterations: int  # the most sweeps any rank ran
    all_converged: bool
    device_ms: float  # the slowest rank's solve
    columns: tuple  # this rank's [lo, hi)
    col_iterations: np.ndarray  # every column, gathered
    col_errors: np.ndarray
    col_converged: np.ndarray


def ppr_batched(graph, degrees, seeds, damping_factor=0.85, threshold=1e-6, max_iters=100, group=None,
                gather=True, stream=None):
    """Personalised PageRank for ``seeds`` with the columns split over the
    ranks of ``group``: every rank holds the whole graph, solves its share of
    the seeds (:func:`even_bounds`) with no exchange between sweeps, and with
    ``gather`` the n x k row-major result is assembled on every rank at the
    end (else each rank returns its n x share block). Returns ``(scores,
    ShardedPprStats)``."""
    import torch
    ex = DistExchange(group)
    k = len(seeds)
    b = even_bounds(k, ex.world)
    lo, hi = int(b[ex.rank]), int(b[ex.rank + 1])
    dev = degrees.device
    local = torch.empty((graph.n, hi - lo), dtype=torch.float32, device=dev)
    st = solve_columns(graph, degrees, seeds, local, b, ex.rank, damping_factor, threshold, max_iters, stream)
    per = torch.zeros((hi - lo, 3), dtype=torch.float64, device=dev)
    if st is not None:
        per[:, 0] = torch.from_numpy(np.asarray(st.col_iterations, np.float64))
        per[:, 1] = torch.from_numpy(np.asarray(st.col_errors, np.float64))
        per[:, 2] = torch.from_numpy(np.asarray(st.col_converged, np.float64))
    counts = np.diff(b)
    per = gather_rows(per, counts, ex).cpu().numpy()
    mx = torch.tensor([st.iterations if st else 0, st.device_ms if st else 0.0,
                       0.0 if (st is None or st.all_converged) else 1.0], dtype=torch.float64, device=dev)
    ex.dist.all_reduce(mx, op=ex.dist.ReduceOp.MAX, group=ex.group)
    mx = mx.cpu().tolist()
    stats = ShardedPprStats(int(mx[0]), mx[2] == 0.0, float(mx[1]), (lo, hi), per[:, 0].astype(np.uint32),
                            per[:, 1].copy(), per[:, 2].astype(bool))
    if not gather:
        return local, stats
    return gather_rows(local.t().contiguous(), counts, ex).t().contiguous(), stats


class ShardedBatch:
    """This rank's graphs of a ragged batch: whole graphs ``[lo, hi)``
    (:func:`graph_bounds`), solved with no exchange between sweeps. The batch
    arrays, in the :class:`~nwgraph_b200.GraphBatch` layout, are passed whole on
    every rank (host arrays or CUDA tensors); the rank keeps a batch of its own
    graphs. :meth:`page_rank` takes and fills this rank's vertices
    (``vertex_range`` of the concatenated per-vertex arrays), and
    :meth:`gather` concatenates every rank's per-vertex results."""

    def __init__(self, vertex_offsets, entry_offsets, row_ptr, col, group=None):
        from .pagerank import GraphBatch
        self.exchange = DistExchange(group)
        self.world, self.rank = self.exchange.world, self.exchange.rank
        vo = np.asarray(vertex_offsets, np.uint64)
        eo = np.asarray(entry_offsets, np.uint64)
        self.bounds = graph_bounds(vo, eo, self.world)
        lo, hi = int(self.bounds[self.rank]), int(self.bounds[self.rank + 1])
        self.graphs = (lo, hi)
        self.vertex_range = (int(vo[lo]), int(vo[hi]))
        self.vertex_counts = [int(vo[self.bounds[q + 1]] - vo[self.bounds[q]]) for q in range(self.world)]
        self.batch = GraphBatch(*batch_slice(vo, eo, row_ptr, col, lo, hi)) if hi > lo else None

    def page_rank(self, degrees, page_rank, damping_factor=0.85, threshold=1e-4, max_iters=20, launch="graph",
                  stream=None):
        """This rank's graphs solved into ``page_rank`` (this rank's vertices);
        its RaggedStats, or None when the rank holds no graph."""
        if self.batch is None:
            return None
        return self.batch.page_rank(degrees, page_rank, damping_factor, threshold, max_iters, launch, stream)

    def gather(self, local):
        """Every rank's per-vertex ``local`` values concatenated in graph order."""
        return gather_rows(local, self.vertex_counts, self.exchange)

    def release(self):
        if self.batch is not None:
            self.batch.release()
