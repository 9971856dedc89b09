"""One rank of the two-rank CPU check of the row-sharded solve.

Launched by tests/test_shard.py through torch.distributed.run with the gloo
backend: each rank builds the CPU stand-in of its shard (tests/oracle_shard.py)
for the same graph, runs nwgraph_b200.shard.run with the torch.distributed
exchange, and writes the ranks and sweep errors it got to <outdir>/rank<r>.npz.
"""
import datetime
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

from nwgraph_b200 import graphs as G, shard as S  # noqa: E402
from oracle_shard import OracleShard  # noqa: E402


def main():
    outdir, thr, iters = sys.argv[1], float(sys.argv[2]), int(sys.argv[3])
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    world, rank = dist.get_world_size(), dist.get_rank()
    g = G.rmat(10, 16, 3)
    deg = g.out_degree()
    bounds, stride = S.shard_bounds(g.row_ptr, world)
    sh = OracleShard(g.row_ptr, g.col, world, rank, bounds, stride)
    out = torch.zeros(g.n, dtype=torch.float32)
    st = S.run([sh], S.DistExchange(), deg, out, 0.85, thr, iters, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    np.savez(os.path.join(outdir, f"rank{rank}.npz"), ranks=out.numpy(), errors=np.array(st.errors),
             iterations=st.iterations, bounds=bounds, stride=stride)


if __name__ == "__main__":
    main()
