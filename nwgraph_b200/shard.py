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
import math
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
        self.dist.all_reduce(l1, op=self.dist.ReduceOp.SUM, group=self.group)
        return float(l1.sum().item())


class LocalExchange:
    """Every shard in this process (their kernels never wait on one another):
    slices are copied into place and the L1 changes summed in rank order."""

    def gather(self, full, slices):
        stride = slices[0].numel()
        for q, s in enumerate(slices):
            full[q * stride:(q + 1) * stride].copy_(s)

    def total(self, l1):
        return math.fsum(l1.cpu().tolist()) if l1.numel() > 1 else float(l1.item())


@dataclass
class ShardedStats:
    iterations: int
    final_error: float
    converged: bool
    device_ms: float
    errors: list = field(default_factory=list)


def run(shards, exchange, degrees, ranks_out, damping=0.85, threshold=1e-4, max_iters=20, device=None):
    """The sharded solve: start, then per sweep (every local shard sweeps,
    the slices are gathered, the L1 changes summed), stop at the first sweep
    whose summed change is < threshold or after max_iters; the ranks are
    gathered and written to ``ranks_out`` (n floats, input order) on every
    rank. ``shards`` are this process's shards in rank order; ``device`` is the
    torch device of the buffers."""
    import torch
    dev = torch.device(device) if device is not None else (ranks_out.device if hasattr(ranks_out, "device") else None)
    stride, world = shards[0].stride, shards[0].world
    on_gpu = dev is not None and dev.type == "cuda"
    stream = torch.cuda.current_stream(dev).cuda_stream if on_gpu else None
    full = torch.zeros(world * stride, dtype=torch.float32, device=dev)
    slices = [torch.zeros(stride, dtype=torch.float32, device=dev) for _ in shards]
    l1 = torch.zeros(len(shards), dtype=torch.float64, device=dev)
    for sh, s in zip(shards, slices):
        sh.start(degrees, s, stream)
    exchange.gather(full, slices)
    if on_gpu:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
    errors = []
    converged = False
    for _ in range(int(max_iters)):
        for j, (sh, s) in enumerate(zip(shards, slices)):
            sh.sweep(full, s, damping, l1[j:j + 1], stream)
        exchange.gather(full, slices)
        e = exchange.total(l1)
        errors.append(e)
        if not math.isfinite(e):
            raise NwgpuError(N.ERR_CUDA, "a bounded device wait gave up on some rank")
        if e < float(threshold):
            converged = True
            break
    ms = 0.0
    if on_gpu:
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
    for sh, s in zip(shards, slices):
        sh.rank_slice(s, stream)
    exchange.gather(full, slices)
    shards[0].unpermute(full, ranks_out, stream)
    if on_gpu:
        torch.cuda.synchronize(dev)
    return ShardedStats(len(errors), errors[-1] if errors else 0.0, converged, ms, errors)


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
