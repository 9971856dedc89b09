"""One rank of the CPU check of batches sharded with no exchange per sweep.

Launched by tests/test_shard.py through torch.distributed.run with the gloo
backend:

* personalised columns: nwgraph_b200.shard.ppr_batched over a CPU stand-in
  graph whose ppr_batched solves each column with the oracle
  (oracle.ppr_jacobi_f32);
* ragged graphs: the rank's graphs (graph_bounds, batch_slice) solved one by
  one with oracle.jacobi_f32, then gathered with gather_rows.

Each rank writes what it got to <outdir>/rank<r>.npz.
"""
import datetime
import os
import sys
from types import SimpleNamespace

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

import oracle as O  # noqa: E402
from nwgraph_b200 import graphs as G, shard as S  # noqa: E402

D, THR, ITERS = 0.85, 1e-6, 100


class OracleColumns:
    """Stand-in for a resident graph: ``ppr_batched`` column by column on the CPU."""

    def __init__(self, g):
        self.g, self.n = g, g.n

    def ppr_batched(self, degrees, seeds, out, damping, threshold, max_iters):
        deg = degrees.numpy().view(np.uint32)
        its, errs, conv = [], [], []
        for c, s in enumerate(np.asarray(seeds)):
            r, it, e = O.ppr_jacobi_f32(self.g.row_ptr, self.g.col, deg, int(s), damping, threshold, max_iters)
            out[:, c] = torch.from_numpy(r)
            its.append(it)
            errs.append(e[-1])
            conv.append(e[-1] < threshold)
        return SimpleNamespace(iterations=max(its), all_converged=all(conv), device_ms=1.0 + dist.get_rank(),
                               col_iterations=np.array(its, np.uint32), col_errors=np.array(errs),
                               col_converged=np.array(conv))


def ppr_case():
    g = G.rmat(9, 8, 5)
    deg = g.out_degree()
    return g, deg, G.random_sources(deg, 7, seed=7)


def ragged_case():
    graphs = [G.rmat(7, 8, 1), G.grid(400), G.rmat(9, 16, 2), G.grid(100), G.rmat(6, 4, 3), G.grid(900),
              G.rmat(8, 8, 4)]
    vo = np.concatenate([[0], np.cumsum([g.n for g in graphs])]).astype(np.uint64)
    eo = np.concatenate([[0], np.cumsum([g.nnz for g in graphs])]).astype(np.uint64)
    return graphs, vo, eo, np.concatenate([g.row_ptr for g in graphs]), np.concatenate([g.col for g in graphs])


def main():
    outdir = sys.argv[1]
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    rank = dist.get_rank()

    g, deg, seeds = ppr_case()
    scores, st = S.ppr_batched(OracleColumns(g), torch.from_numpy(deg.view(np.int32)), seeds, D, THR, ITERS)
    block, _ = S.ppr_batched(OracleColumns(g), torch.from_numpy(deg.view(np.int32)), seeds, D, THR, ITERS,
                             gather=False)

    graphs, vo, eo, rp, cl = ragged_case()
    ex = S.DistExchange()
    b = S.graph_bounds(vo, eo, ex.world)
    lo, hi = int(b[rank]), int(b[rank + 1])
    svo, seo, srp, scl = S.batch_slice(vo, eo, rp, cl, lo, hi)
    local = []
    for j in range(hi - lo):
        grp = srp[int(svo[j]) + j:int(svo[j + 1]) + j + 1]
        gcl = scl[int(seo[j]):int(seo[j + 1])]
        r, _, _ = O.jacobi_f32(grp, gcl, O.out_degree(grp, gcl, len(grp) - 1), D, THR, 200)
        local.append(r)
    local = torch.from_numpy(np.concatenate(local) if local else np.zeros(0, np.float32))
    counts = [int(vo[b[q + 1]] - vo[b[q]]) for q in range(ex.world)]
    ragged = S.gather_rows(local, counts, ex)

    dist.barrier()
    dist.destroy_process_group()
    np.savez(os.path.join(outdir, f"rank{rank}.npz"), scores=scores.numpy(), block=block.numpy(),
             columns=np.array(st.columns), iterations=st.iterations, all_converged=st.all_converged,
             device_ms=st.device_ms, col_iterations=st.col_iterations, col_errors=st.col_errors,
             col_converged=st.col_converged, ragged=ragged.numpy(), graph_bounds=b)


if __name__ == "__main__":
    main()
