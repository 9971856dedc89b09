"""CPU stand-in for one rank's GPU shard -- TEST INFRASTRUCTURE ONLY.

It has GpuShard's methods (start, sweep, decide, rank_slice, unpermute) and the same
layout: the whole graph relabelled by descending row length (stably), this
rank's internal rows [bounds[rank], bounds[rank+1]), column ids mapped to the
padded all-gather layout (rank q's rows at q * stride). Each row is summed
sequentially in FP32, as page_rank_v10 does (experimental/algorithms/
page_rank.hpp:409-423), so a sharded run must give the same ranks bit for bit
as a one-shard run, whatever the partition; that is what the multi-rank tests
check on CPU, with the exchange going through torch.distributed (gloo).
"""
import numpy as np


class OracleShard:
    def __init__(self, row_ptr, col, world, rank, bounds, stride):
        rp = np.asarray(row_ptr, np.int64)
        cl = np.asarray(col, np.int64)
        n = len(rp) - 1
        lens = np.diff(rp)
        inv = np.argsort(-lens, kind="stable")          # internal id -> input id
        perm = np.empty(n, np.int64)
        perm[inv] = np.arange(n)                        # input id -> internal id
        bounds = np.asarray(bounds, np.int64)
        lo, hi = int(bounds[rank]), int(bounds[rank + 1])
        owner = np.searchsorted(bounds, np.arange(n), side="right") - 1
        pos_of_internal = owner * stride + (np.arange(n) - bounds[owner])
        rows = inv[lo:hi]
        self.lens = lens[rows]
        self.lrp = np.concatenate([[0], np.cumsum(self.lens)])
        self.lcol = np.concatenate([pos_of_internal[perm[cl[rp[r]:rp[r + 1]]]] for r in rows] + [np.zeros(0, np.int64)])
        self.inv_local = rows
        self.pos_of_input = pos_of_internal[perm]
        self.n, self.world, self.rank, self.stride = n, world, rank, stride
        self.rows = hi - lo
        self.rank_v = np.zeros(self.rows, np.float32)
        self.deg = np.ones(self.rows, np.uint32)

    def start(self, degrees, contrib_slice, stream=None):
        self.deg = np.asarray(degrees, np.uint32)[self.inv_local]
        self.rank_v = np.full(self.rows, np.float32(1.0 / self.n), np.float32)
        self.stopped, self.last_l1 = False, 0.0
        out = contrib_slice.numpy()
        with np.errstate(divide="ignore"):
            out[: self.rows] = self.rank_v / self.deg.astype(np.float32)

    def sweep(self, contrib_all, contrib_slice, damping, l1, stream=None):
        if self.stopped:  # nwgpu_shard_sweep after nwgpu_shard_decide stopped the solve: nothing changes
            l1.numpy()[0] = self.last_l1
            return
        full = contrib_all.numpy()
        vals = full[self.lcol]
        z = np.zeros(self.rows, np.float32)
        for k in range(int(self.lens.max()) if self.rows else 0):  # sequential FP32 row sums
            r = np.nonzero(self.lens > k)[0]
            z[r] += vals[self.lrp[r] + k]
        base = np.float32((1.0 - float(damping)) / self.n)
        nr = (np.float64(np.float32(damping)) * z.astype(np.float64) + np.float64(base)).astype(np.float32)
        self.last_l1 = float(np.abs(nr.astype(np.float64) - self.rank_v.astype(np.float64)).sum())
        l1.numpy()[0] = self.last_l1
        self.rank_v = nr
        with np.errstate(divide="ignore"):
            contrib_slice.numpy()[: self.rows] = nr / self.deg.astype(np.float32)

    def decide(self, total, threshold, max_iters, state, errors, errors_cap, stream=None):
        """nwgpu_shard_decide restated: state = {sweeps decided, stopped, converged, failed}."""
        st = state.numpy()
        if st[1]:
            return
        e = float(total.numpy()[0])
        if errors is not None and st[0] < errors_cap:
            errors.numpy()[st[0]] = e
        failed = e != e
        conv = (not failed) and e < float(threshold)
        st[0] += 1
        if conv or failed or st[0] >= int(max_iters):
            st[1], st[2], st[3] = 1, int(conv), int(failed)
            self.stopped = True

    def rank_slice(self, out, stream=None):
        out.numpy()[: self.rows] = self.rank_v

    def unpermute(self, ranks_all, ranks, stream=None):
        ranks.numpy()[:] = ranks_all.numpy()[self.pos_of_input]
