"""Benchmark: FP32 PageRank on a scale-24 RMAT graph, one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the configuration the headline metric is quoted on): RMAT scale 24
(16.8M vertices), edge factor 16, a/b/c/d = .57/.19/.19/.05, symmetrised and
deduplicated (~5.3e8 directed entries), uint32 CSR in NWGraph's adjacency<1>
layout, damping 0.85, 20 fixed sweeps (threshold 0), FP32 scores. One step =
one full solve. Inputs are seeded synthetic (the reference's GAP datasets are
not available here); col[] alone (2.1 GB) is far larger than L2, so no L2
flush is needed between steps.

Our arm prints one JSON line with
  value     GTEPS per sweep (nnz / sweep time) over K solves with the CSR and
            degrees resident in HBM, CUDA events on the launching stream,
            max over ranks;
  e2e       the same metric through the public API with pinned HOST buffers:
            graph upload + validation + tiling, the solve, ranks back to host;
  roofline  the sweep kernel against the measured HBM copy bandwidth, with the
            graded bytes per sweep 4 nnz + 4 (n+1) + 20 n;
  cpu_baseline  NWGraph's page_rank (v11) compiled from its headers at its
            release flags, timed on this host's cores on a 2-sweep sample.
With --gpus N (torchrun) every rank solves its own resident replica
(weak scaling, no data-path collective: the headline), and the row-sharded
solve of the one graph across the ranks is timed beside it (strong scaling,
key row_sharded: an all-gather of contributions and an all-reduce of the L1
change per sweep over NCCL, the stopping decision taken on the device).

--impl reference runs NWGraph's own page_rank on this host's CPU cores
(rank 0 only), each step a 2-sweep sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PR GTEPS/iter & %HBM roofline; batched PPR vs looped plain at 1e-6 L1; bwd/fwd"
UNIT = "GTEPS"
DAMPING = 0.85
SWEEPS = 20
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--edge-factor", type=float, default=16)
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-sample-sweeps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-relabel", action="store_true", help="keep the input vertex order on the device")
    ap.add_argument("--no-shard", action="store_true",
                    help="skip the row-sharded solve of the one graph across the ranks (all-gather over NCCL each "
                         "sweep, stopping decided on the device), timed by default next to the replica headline")
    ap.add_argument("--no-autotune", action="store_true",
                    help="default launch settings instead of the tuned ones (tuning runs at graph creation)")
    ap.add_argument("--ppr-scale", type=int, default=22, help="graph scale of the batched-PPR comparison (0: skip)")
    ap.add_argument("--ppr-k", type=int, default=64)
    ap.add_argument("--ragged-graphs", type=int, default=4096,
                    help="graphs of the ragged-batch comparison (0: skip)")
    ap.add_argument("--ragged-max-n", type=float, default=1e6, help="largest graph of the ragged batch")
    ap.add_argument("--vjp-scale", type=int, default=20,
                    help="graph scale of the weighted forward vs adjoint (backward) timing (0: skip)")
    ap.add_argument("--launch", default="graph", choices=["graph", "stream"],
                    help="sweep loop as a CUDA graph with a device-side while loop, or one launch per sweep")
    return ap.parse_args()


def max_over_ranks(values, dist=None, device="cpu"):
    """Element-wise maximum over ranks of a few timings. Every rank calls it
    the same number of times, in the same order (one all-reduce each)."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def job_gteps(world, nnz, sweeps, ms_per_step):
    """Whole-job throughput: every rank solves its own replica of nnz entries
    for `sweeps` sweeps per step; the step time is the slowest rank's."""
    return world * nnz * sweeps / (ms_per_step * 1e-3) / 1e9


def graded_bytes(n, nnz):
    return 4.0 * nnz + 4.0 * (n + 1) + 20.0 * n


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def gather_ceiling(log2_len=24, iters=256, reps=5):
    """The measured ceiling of random 4-byte L2 gathers on this GPU
    (libnwprobe.so): the sweep's cold-gather load form, 8 in flight per thread,
    one 1024-thread CTA per SM, uniform random indices into a 2^log2_len-float
    (64 MB) L2-resident table. Returns loads per second."""
    import ctypes as C
    lib = C.CDLL(os.path.join(ROOT, "nwgraph_b200", "libnwprobe.so"))
    rate, ms = C.c_double(), C.c_double()
    rc = lib.nwprobe_gather_rate(C.c_uint32(log2_len), C.c_uint32(iters), C.c_uint32(reps), C.byref(rate),
                                 C.byref(ms))
    if rc:
        raise RuntimeError(f"gather probe failed: cudaError {rc}")
    return rate.value


def hub_tier_counts(rp_d, cl_d, thresholds):
    """Entries whose column, in the engine's internal ids (vertices by
    descending row length, stably), is >= each threshold: the gathers that
    leave the shared-memory hub table and the L1 tier in every sweep."""
    import torch
    ln = (rp_d[1:] - rp_d[:-1]).long()
    order = torch.sort(-ln, stable=True).indices
    newid = torch.empty(ln.numel(), dtype=torch.int32, device=ln.device)
    newid[order] = torch.arange(ln.numel(), dtype=torch.int32, device=ln.device)
    del ln, order
    counts = [0] * len(thresholds)
    step = 1 << 26
    for s in range(0, cl_d.numel(), step):
        ids = newid[cl_d[s:s + step].long()]
        for j, t in enumerate(thresholds):
            counts[j] += int((ids >= t).sum())
    return counts


def sweep_traffic_per_launch(args, sweep):
    """DRAM bytes per launch of this workload's sweep kernel (``sweep``:
    "blocked" or "binned") from roofline_traffic.json (one ncu capture of the
    benchmark command), or None without a capture."""
    workload = f"rmat{args.scale}_ef{int(args.edge_factor)}_pagerank_f32"
    try:
        with open(os.path.join(ROOT, "roofline_traffic.json")) as f:
            entries = json.load(f)["entries"]
    except (OSError, ValueError, KeyError):
        return None
    for e in entries:
        if (e.get("workload") == workload and bool(e.get("relabel")) == (not args.no_relabel)
                and e.get("sweep") == sweep):
            return float(e["traffic_bytes_per_launch"])
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()  # nvidia-smi takes a moment to start: the timed region waits for its first sample
            while not self.out and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def make_graph(args, device=False):
    """The RMAT workload graph: built on the GPU (nwgpu_rmat_edges +
    nwgpu_csr_from_edges) for our arm, on the host for the reference arm;
    both give the same CSR bit for bit (tests/test_construct_gpu.py)."""
    t0 = time.time()
    if device:
        from nwgraph_b200 import construct as K
        g = K.rmat(args.scale, args.edge_factor, args.seed)
    else:
        from nwgraph_b200 import graphs as G
        g = G.rmat(args.scale, args.edge_factor, args.seed)
    return g, g.out_degree(), time.time() - t0


def cpu_reference_sample(g, deg, sweeps, nthreads):
    """NWGraph page_rank v11 at its release flags on this host (oracle/_ref),
    or the C restatement of page_rank_v10 when the reference build is absent."""
    import oracle as O
    if O.ref_available(fast=True):
        rg = O.RefGraph(g.row_ptr, g.col, deg, fast=True)
        _, it, _, secs = rg.page_rank(11, DAMPING, 0.0, sweeps, nthreads)
        # the configuration's threshold-1e-4 run on the reference: both solvers' sweep counts
        _, it11, e11, _ = rg.page_rank(11, DAMPING, 1e-4, 1000, nthreads)
        _, it10, _, _ = rg.page_rank(10, DAMPING, 1e-4, 1000, nthreads)
        rg.close()
        t = float(np.mean(secs))
        return {"value": g.nnz / t / 1e9, "unit": UNIT, "cores": nthreads, "kind": "reference",
                "sample": f"{it} sweeps of nw::graph::page_rank (v11, -Ofast, TBB-API shim) on the full graph; "
                          f"mean sweep {t * 1e3:.1f} ms from the reference's own trace",
                "threshold_1e-4_sweeps": {"page_rank_v11": it11, "page_rank_v10": it10, "threads": nthreads,
                                          "v11_last_error": float(e11[-1]) if len(e11) else None}}
    t0 = time.perf_counter()
    O.jacobi_f32(g.row_ptr, g.col, deg, DAMPING, 0.0, 1)
    t = time.perf_counter() - t0
    return {"value": g.nnz / t / 1e9, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "1 sweep of the C restatement of page_rank_v10 on the full graph (includes init)"}


def ppr_batched_vs_looped(scale, k, stream, dist=None, launch="graph"):
    """Batched personalised PageRank (k one-hot seeds drawn among vertices with
    out-degree >= 1, per-column L1 < 1e-6, at most 100 sweeps) against k
    looped single-seed solves on the same engine, all resident in HBM. Over
    several ranks each solves its share of the seeds (even_bounds) with no
    exchange, and the times are the slowest rank's."""
    import torch
    from nwgraph_b200 import Graph, graphs as G, shard as S
    g = G.rmat(scale, 16, 42)
    deg = g.out_degree()
    world, rank = (dist.get_world_size(), dist.get_rank()) if dist else (1, 0)
    cb = S.even_bounds(k, world)
    seeds = G.random_sources(deg, k, seed=7)[cb[rank]:cb[rank + 1]]
    k_all, k = k, int(cb[rank + 1] - cb[rank])
    dev = torch.device("cuda")
    rp = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    cl = torch.from_numpy(g.col.view(np.int32)).to(dev)
    dg = torch.from_numpy(deg.view(np.int32)).to(dev)
    out_b = torch.empty((g.n, k), dtype=torch.float32, device=dev)
    out_1 = torch.empty(g.n, dtype=torch.float32, device=dev)
    with Graph(rp, cl) as h:
        h.ppr_batched(dg, seeds, out_b, DAMPING, 1e-6, 100, stream=stream, launch=launch)  # warm-up
        h.ppr(dg, int(seeds[0]), out_1, DAMPING, 1e-6, 100, stream=stream, launch=launch)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        stb = h.ppr_batched(dg, seeds, out_b, DAMPING, 1e-6, 100, stream=stream, launch=launch)
        e1.record(stream)
        torch.cuda.synchronize()
        t_batched = e0.elapsed_time(e1)
        looped_sweeps = 0
        e0.record(stream)
        for c in range(k):
            st = h.ppr(dg, int(seeds[c]), out_1, DAMPING, 1e-6, 100, stream=stream, launch=launch)
            looped_sweeps += st.iterations
        e1.record(stream)
        torch.cuda.synchronize()
        t_looped = e0.elapsed_time(e1)
        worst = 0.0  # equal accuracy: sampled columns of both agree (checked after timing)
        for c in range(0, k, 8):
            h.ppr(dg, int(seeds[c]), out_1, DAMPING, 1e-6, 100, stream=stream)
            worst = max(worst, float((out_1 - out_b[:, c]).abs().max()))
    t_batched, t_looped, worst, b_sweeps, not_conv = max_over_ranks(
        [t_batched, t_looped, worst, stb.iterations, 0.0 if stb.all_converged else 1.0], dist, dev)
    if dist:  # whole-job sweep count of the looped solves
        tot = torch.tensor([float(looped_sweeps)], dtype=torch.float64, device=dev)
        dist.all_reduce(tot)
        looped_sweeps = int(tot.item())
    return {"graph": f"rmat{scale}_ef16", "n": g.n, "nnz": g.nnz, "k": k_all, "threshold": 1e-6,
            "columns_per_rank": np.diff(cb).tolist(),
            "batched_ms": t_batched, "looped_ms": t_looped, "speedup": t_looped / t_batched,
            "batched_sweeps": int(b_sweeps), "looped_sweeps_total": looped_sweeps,
            "all_converged": not_conv == 0.0, "max_abs_batched_vs_looped": worst}


def ragged_vs_looped(num_graphs, max_n, stream, sample_mod=16, dist=None):
    """One ragged-batch solve of every graph (per-graph L1 < 1e-6, at most 200
    sweeps) against looped single-graph solves on the same engine, timed on a
    sample (graph ids = 0 or 1 mod sample_mod: RMAT and grid alike) and
    scaled to the batch. Over several ranks each builds and solves its own
    whole graphs (weighted_bounds over the expected rows plus entries) with no
    exchange; times are the slowest rank's, counts are summed."""
    import torch
    from nwgraph_b200 import Graph, construct as K, shard as S
    world, rank = (dist.get_world_size(), dist.get_rank()) if dist else (1, 0)
    ns, efs = K.ragged_sizes(num_graphs, max_n)
    ids = np.arange(num_graphs)
    gb = S.weighted_bounds(np.where(ids % 2 == 0, ns * (1 + 2 * efs), 5 * ns), world)
    mine = range(int(gb[rank]), int(gb[rank + 1]))
    t0 = time.time()
    parts, degs = K.ragged_graphs(num_graphs, max_n, graphs=mine)
    torch.cuda.synchronize()
    build_s = time.time() - t0
    nv = sum(int(p[0].numel()) - 1 for p in parts)
    nnz = sum(int(p[1].numel()) for p in parts)
    sample = [j for j, g in enumerate(mine) if g % sample_mod in (0, 1)]
    kept = [(parts[j][0].clone(), parts[j][1].clone(), degs[j].clone()) for j in sample]
    b, deg = K.batch_from_device_csrs(parts, degs)
    out = torch.empty(max(b.n, 1), dtype=torch.float32, device="cuda")
    b.page_rank(deg, out, DAMPING, 1e-6, 200, stream=stream)  # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    st = b.page_rank(deg, out, DAMPING, 1e-6, 200, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    t_batched = e0.elapsed_time(e1)
    b.release()
    del out, deg, b
    looped_ms, looped_swept = 0.0, 0.0
    for rp, cl, dg in kept:
        with Graph(rp, cl) as h:
            o = torch.empty(rp.numel() - 1, dtype=torch.float32, device="cuda")
            h.page_rank(dg, o, DAMPING, 1e-6, 200, stream=stream)  # warm-up
            torch.cuda.synchronize()
            e0.record(stream)
            s1 = h.page_rank(dg, o, DAMPING, 1e-6, 200, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
            looped_ms += e0.elapsed_time(e1)
            looped_swept += float(cl.numel()) * s1.iterations
    scale = len(mine) / max(len(sample), 1)
    looped_ms *= scale
    swept, conv = st.entries_swept, st.converged_graphs
    med = int(np.median(st.graph_iterations))
    if dist:
        dev = torch.device("cuda", torch.cuda.current_device())
        sums = torch.tensor([nv, nnz, swept, conv], dtype=torch.float64, device=dev)
        dist.all_reduce(sums, group=None)
        nv, nnz, swept, conv = (int(sums[0]), int(sums[1]), float(sums[2]), int(sums[3]))
        t_batched, looped_ms, build_s = max_over_ranks([t_batched, looped_ms, build_s], dist, dev)
    return {"graphs": num_graphs, "graphs_per_rank": np.diff(gb).tolist(), "n_range": [1000, int(max_n)],
            "vertices": nv, "entries": nnz,
            "threshold": 1e-6, "max_iters": 200, "build_s": build_s, "batched_ms": t_batched,
            "batched_sweeps_rank0": st.sweeps, "converged_graphs": conv, "graph_sweeps_median_rank0": med,
            "entries_swept": swept, "batched_gteps": swept / (t_batched * 1e6),
            "looped_ms_est": looped_ms, "looped_sample": f"graph ids 0, 1 mod {sample_mod} of each rank's "
            f"graphs, summed and scaled to the rank's graphs (x{scale:g} on rank 0)",
            "speedup_est": looped_ms / t_batched}


def vjp_vs_forward(scale, stream):
    """Weighted PageRank forward and its implicit-adjoint backward on RMAT
    `scale` (weights U(0.1, 1) seed 1234, uniform teleport, L = c . r with
    c ~ N(0,1) seed 99). Each side runs to an FP64 L1 change of 1e-6 times its
    own scale (1 for the ranks, sum |c| for the adjoint). Times with CUDA
    events on `stream`."""
    import torch
    from nwgraph_b200 import Graph, graphs as G
    g = G.rmat(scale, 16, 42)
    dev = stream.device
    w = torch.from_numpy(G.edge_weights(g.nnz, seed=1234)).to(dev)
    c = torch.from_numpy(np.random.default_rng(99).standard_normal(g.n).astype(np.float32)).to(dev)
    rp = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    cl = torch.from_numpy(g.col.view(np.int32)).to(dev)
    r = torch.empty(g.n, dtype=torch.float32, device=dev)
    dw = torch.empty(g.nnz, dtype=torch.float32, device=dev)
    dt = torch.empty(g.n, dtype=torch.float32, device=dev)
    thr_b = 1e-6 * float(c.abs().sum())
    with Graph(rp, cl, weights=w) as h:
        fwd = lambda: h.weighted_page_rank(None, r, DAMPING, 1e-6, 1000, stream=stream)  # noqa: E731
        bwd = lambda: h.page_rank_vjp(r, c, dw, dt, DAMPING, thr_b, 1000, stream=stream)  # noqa: E731
        for _ in range(2):
            fwd()
            bwd()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        e[0].record(stream)
        sf = fwd()
        e[1].record(stream)
        sb = bwd()
        e[2].record(stream)
        torch.cuda.synchronize()
    t_f, t_b = e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])
    return {"graph": f"rmat{scale}_ef16_weighted", "n": g.n, "nnz": g.nnz, "forward_ms": t_f, "backward_ms": t_b,
            "bwd_over_fwd": t_b / t_f, "forward_sweeps": sf.iterations, "adjoint_sweeps": sb.iterations,
            "forward_ms_per_sweep": sf.ms_per_iter, "adjoint_ms_per_sweep": sb.ms_per_iter,
            "backward_includes": "adjoint solve on the out-row CSR + dL/dw (nnz) + dL/dt (n)"}


def row_sharded(g, deg, dev, dist, steps):
    """The row-sharded solve (nwgraph_b200.shard) of the whole graph: 20
    fixed sweeps per step, each followed by the all-gather of the ranks'
    contribution slices and the all-reduce of their L1 changes (one shard and
    plain copies on one GPU). Strong scaling: every rank holds 1/N of the rows."""
    import torch
    from nwgraph_b200 import shard as S
    rp = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    cl = torch.from_numpy(g.col.view(np.int32)).to(dev)
    dg = torch.from_numpy(deg.view(np.int32)).to(dev)
    out = torch.empty(g.n, dtype=torch.float32, device=dev)
    if dist:
        sg = S.ShardedGraph(rp, cl)
        solve = lambda: sg.page_rank(dg, out, DAMPING, 0.0, SWEEPS)  # noqa: E731
        world, bounds = sg.world, sg.bounds
    else:
        bounds, stride = S.shard_bounds(g.row_ptr, 1)
        sh = S.GpuShard(rp, cl, 1, 0, bounds, stride)
        solve = lambda: S.run([sh], S.LocalExchange(), dg, out, DAMPING, 0.0, SWEEPS, device=dev)  # noqa: E731
        world = 1
    del rp, cl
    for _ in range(3):
        solve()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        solve()
    e1.record()
    torch.cuda.synchronize()
    ms, = max_over_ranks([e0.elapsed_time(e1) / steps], dist, dev)
    return {"world": world, "ms_per_step": ms, "ms_per_sweep": ms / SWEEPS,
            "gteps": g.nnz * SWEEPS / (ms * 1e-3) / 1e9, "scaling": "strong",
            "rows_per_rank": np.diff(np.asarray(bounds, np.int64)).tolist(),
            "exchange": "all_gather_into_tensor + all_reduce (NCCL)" if dist else "one shard, copies"}


def wppr_batched_vs_looped(scale, k, stream):
    """The weighted configuration's batched variant: k teleport vectors
    (random distributions, seed 99) on the RMAT graph with weights U(0.1, 1)
    (seed 1234), per-column L1 < 1e-6, against k looped weighted solves."""
    import torch
    from nwgraph_b200 import Graph, graphs as G
    g = G.rmat(scale, 16, 42)
    w = G.edge_weights(g.nnz, seed=1234)
    t = np.random.default_rng(99).uniform(0.0, 1.0, (g.n, k))
    t = (t / t.sum(axis=0, keepdims=True)).astype(np.float32)
    dev = torch.device("cuda")
    td = torch.from_numpy(t).to(dev)
    cols = [td[:, c].contiguous() for c in range(k)]
    out = torch.empty((g.n, k), dtype=torch.float32, device=dev)
    out1 = torch.empty(g.n, dtype=torch.float32, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Graph(g.row_ptr, g.col, weights=w) as h:
        h.weighted_page_rank_batched(td, out, DAMPING, 1e-6, 300, stream=stream)  # warm-up (out-row CSR, buffers)
        h.weighted_page_rank(cols[0], out1, DAMPING, 1e-6, 300, stream=stream)
        torch.cuda.synchronize()
        e0.record(stream)
        sb = h.weighted_page_rank_batched(td, out, DAMPING, 1e-6, 300, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        t_b = e0.elapsed_time(e1)
        sweeps = 0
        e0.record(stream)
        for c in range(k):
            sweeps += h.weighted_page_rank(cols[c], out1, DAMPING, 1e-6, 300, stream=stream).iterations
        e1.record(stream)
        torch.cuda.synchronize()
        t_l = e0.elapsed_time(e1)
        worst = float((out1 - out[:, k - 1]).abs().max())
    return {"graph": f"rmat{scale}_ef16_weighted", "n": g.n, "nnz": g.nnz, "k": k, "threshold": 1e-6,
            "batched_ms": t_b, "looped_ms": t_l, "speedup": t_l / t_b, "batched_sweeps": sb.iterations,
            "looped_sweeps_total": sweeps, "all_converged": sb.all_converged,
            "max_abs_batched_vs_looped_last_column": worst}


class _HostCsr:
    def __init__(self, row_ptr, col):
        self.row_ptr, self.col = row_ptr, col
        self.n, self.nnz = len(row_ptr) - 1, int(row_ptr[-1])


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    nthreads = os.cpu_count() or 1
    import oracle as O
    kind = "reference" if O.ref_available(fast=True) else "port"
    if kind == "reference":
        # the input from the builder copy inside the reference library: this arm maps none of the engine's
        g = _HostCsr(*O.ref_rmat(args.scale, args.edge_factor, args.seed))
        deg = np.bincount(g.col, minlength=g.n).astype(np.uint32)
    else:
        g, deg, _ = make_graph(args)
    if kind == "reference":
        rg = O.RefGraph(g.row_ptr, g.col, deg, fast=True)
        run = lambda: rg.page_rank(11, DAMPING, 0.0, args.cpu_sample_sweeps, nthreads)[3]  # noqa: E731
    else:
        run = lambda: np.array([_time_port(g, deg)])  # noqa: E731
    for _ in range(args.warmup):
        run()
    secs = np.concatenate([run() for _ in range(args.steps)])
    t = float(np.mean(secs))
    value = g.nnz / t / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3 * args.cpu_sample_sweeps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"rmat{args.scale}_ef{int(args.edge_factor)}_pagerank_f32", "n": g.n, "nnz": g.nnz,
                   "sweeps_per_step": args.cpu_sample_sweeps, "damping": DAMPING},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads if kind == "reference" else 1, "kind": kind,
                         "sample": f"{args.steps} steps x {args.cpu_sample_sweeps} sweeps of nw::graph::page_rank "
                                   f"(v11) on the full graph, sweep times from its own trace"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _time_port(g, deg):
    import oracle as O
    t0 = time.perf_counter()
    O.jacobi_f32(g.row_ptr, g.col, deg, DAMPING, 0.0, 1)
    return time.perf_counter() - t0


def launches_per_step(args):
    """Kernels one timed step launches: degrees to internal order (relabelled
    graphs), rank init, two per sweep (the sweep kernel and its finishing
    kernel, on the binned and the merge-path sweep alike), the CUDA graph's
    arm kernel, ranks back to input order (relabelled graphs)."""
    return SWEEPS * 2 + 1 + (1 if args.launch == "graph" else 0) + (2 if not args.no_relabel else 0)


def run_ours(args):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    from nwgraph_b200 import Graph
    g, deg, gen_s = make_graph(args, device=True)
    n, nnz = g.n, g.nnz
    B = graded_bytes(n, nnz)
    stream = torch.cuda.current_stream(dev)

    # ---- resident: CSR + degrees in HBM ------------------------------------
    rp_d = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    cl_d = torch.from_numpy(g.col.view(np.int32)).to(dev)
    deg_d = torch.from_numpy(deg.view(np.int32)).to(dev)
    out_d = torch.empty(n, dtype=torch.float32, device=dev)
    h = Graph(rp_d, cl_d, relabel=not args.no_relabel, autotune=not args.no_autotune)
    info0 = h.info()
    # the random-gather ceiling bounds the binned sweep (row order); the blocked sweep reads its gathers in
    # source order and is bounded by the DRAM stream of its entries instead
    tiers = (hub_tier_counts(rp_d, cl_d, [info0["hub_smem_ids"], info0["hub_l1_ids"]])
             if info0["binned"] and info0["hub_l1_ids"] and not info0["blocked"] else None)
    del rp_d, cl_d
    torch.cuda.empty_cache()
    for _ in range(max(args.warmup, 3)):
        h.page_rank(deg_d, out_d, DAMPING, 0.0, SWEEPS, stream=stream, launch=args.launch)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    sweep_ms, iters = 0.0, 0
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            st = h.page_rank(deg_d, out_d, DAMPING, 0.0, SWEEPS, stream=stream, launch=args.launch)
            sweep_ms += st.device_ms
            iters += st.iterations
        e1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    total_ms, t_sweep_ms = max_over_ranks([e0.elapsed_time(e1), sweep_ms / max(iters, 1)], dist, dev)
    ms_per_step = total_ms / args.steps
    value = job_gteps(world, nnz, SWEEPS, ms_per_step)
    # threshold-1e-4 run (config: "20 fixed iterations plus a threshold-1e-4 run")
    st_thr = h.page_rank(deg_d, out_d, DAMPING, 1e-4, 1000, stream=stream, launch=args.launch)

    # ---- end to end through the public API with pinned host buffers ---------
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
    rp_h, cl_h, deg_h = pin(g.row_ptr), pin(g.col), pin(deg)
    out_h = torch.empty(n, dtype=torch.float32).pin_memory().numpy()
    e2e_steps = max(1, args.e2e_steps)

    def e2e_step():
        with Graph(rp_h, cl_h, relabel=not args.no_relabel, autotune=not args.no_autotune) as hh:
            hh.page_rank(deg_h, out_h, DAMPING, 0.0, SWEEPS, launch=args.launch)

    e2e_step()  # warm-up (context, allocator)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    w0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    f1.record(stream)
    torch.cuda.synchronize()
    wall_e2e = (time.perf_counter() - w0) / e2e_steps
    e2e_ms, = max_over_ranks([f0.elapsed_time(f1) / e2e_steps], dist, dev)
    e2e_value = job_gteps(world, nnz, SWEEPS, e2e_ms)

    info = h.info()
    h.release()
    del rp_h, cl_h, deg_h, out_h
    ppr = (ppr_batched_vs_looped(args.ppr_scale, args.ppr_k, stream, dist, launch=args.launch)
           if args.ppr_scale > 0 else None)
    vjp = vjp_vs_forward(args.vjp_scale, stream) if args.vjp_scale > 0 else None
    wppr = wppr_batched_vs_looped(args.vjp_scale, 16, stream) if args.vjp_scale > 0 else None
    ragged = (ragged_vs_looped(args.ragged_graphs, args.ragged_max_n, stream, dist=dist)
              if args.ragged_graphs > 0 else None)
    sharded = row_sharded(g, deg, dev, dist, args.steps) if not args.no_shard else None

    peak, peak_kind = peaks()
    achieved = B / (t_sweep_ms * 1e-3) / 1e9
    gather_roof = None
    if tiers:
        ceiling = gather_ceiling()
        l2_rate = tiers[1] / (t_sweep_ms * 1e-3)
        gather_roof = {"bound": "random 4-byte L2 gathers", "achieved": l2_rate / 1e9, "peak": ceiling / 1e9,
                       "unit": "G loads/s", "frac": l2_rate / ceiling, "l2_loads_per_sweep": tiers[1],
                       "loads_past_shared_memory_per_sweep": tiers[0],
                       # counting the L1-tier loads as requests too (an upper bound on the request rate)
                       "frac_past_shared_memory": tiers[0] / (t_sweep_ms * 1e-3) / ceiling,
                       "peak_how": "libnwprobe.so on this GPU: the sweep's cold-gather load, 8 in flight per thread, "
                                   "one 1024-thread CTA per SM, random indices into a 64 MB L2-resident table"}
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_reference_sample(g, deg, args.cpu_sample_sweeps, os.cpu_count() or 1)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"rmat{args.scale}_ef{int(args.edge_factor)}_pagerank_f32", "n": n, "nnz": nnz,
                   "sweeps_per_step": SWEEPS, "threshold": 0.0, "damping": DAMPING,
                   "l2": "inputs larger than L2 (col 4*nnz bytes), no flush", "parallelism": f"replicas{world}",
                   "tile_items": info["tile_items"], "grid": info["grid"], "num_tiles": info["num_tiles"],
                   "launch": args.launch, "relabel": not args.no_relabel,
                   "sweep": {k: info[k] for k in ("blocked", "block_count", "block_items", "block_loads",
                                                  "block_piece_entries", "binned",
                                                  "sweep_threads", "sweep_grid", "hub_smem_ids",
                                                  "hub_l1_ids", "long_row_entries", "chunk_entries", "bin0_rows_per_warp", "tuned",
                                                  "tuned_us_per_sweep")}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": sweep_traffic_per_launch(args, "blocked" if info["blocked"] else "binned"),
                     "peak_kind": peak_kind,
                     "bytes_per_sweep": B, "sweep_ms": t_sweep_ms},
        "gather_roofline": gather_roof,
        "gteps_per_sweep_kernel": nnz / (t_sweep_ms * 1e-3) / 1e9,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(4 * (n + 1) + 4 * nnz + 4 * n),
                "d2h_bytes_per_step": int(4 * n), "ms_per_step": e2e_ms, "wall_ms_per_step": wall_e2e * 1e3,
                "includes": "H2D of row_ptr+col+degrees, device validation + tiling, 20 sweeps, D2H of ranks"},
        "threshold_run": {"threshold": 1e-4, "sweeps": st_thr.iterations, "converged": st_thr.converged,
                          "device_ms": st_thr.device_ms},
        "gpu_launches": args.steps * launches_per_step(args),
        "clocks": clk.summary(),
        "graph_gen_s": gen_s,
    }
    if ppr:
        line["ppr_batched_vs_looped"] = ppr
    if vjp:
        line["vjp_vs_forward"] = vjp
    if wppr:
        line["wppr_batched_vs_looped"] = wppr
    if ragged:
        line["ragged_batch_vs_looped"] = ragged
    if sharded:
        line["row_sharded"] = sharded
    if cpu:
        ref_counts = cpu.pop("threshold_1e-4_sweeps", None)
        if ref_counts:
            line["threshold_run"]["reference"] = ref_counts
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
