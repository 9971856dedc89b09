"""One rank of the two-rank CPU check of bench.py's multi-rank host logic.

Launched by tests/test_multirank.py through torch.distributed.run, the way
bench.py is launched for N > 1, but with the gloo backend: each rank reports
per-rank timings that differ, takes the maximum over ranks with bench's own
helper, and writes what it got to <outdir>/rank<r>.json.
"""
import datetime
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import torch.distributed as dist  # noqa: E402

import bench  # noqa: E402


def main():
    rank = int(os.environ["RANK"])
    world = int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    # the step timings of bench.run_ours: total and per-sweep, then e2e
    total, sweep = bench.max_over_ranks([100.0 + 10.0 * rank, 2.0 - 0.5 * rank], dist)
    e2e, = bench.max_over_ranks([50.0 * (rank + 1)], dist)
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(sys.argv[1], f"rank{rank}.json"), "w") as f:
        json.dump({"rank": rank, "world": world, "total": total, "sweep": sweep, "e2e": e2e,
                   "gteps": bench.job_gteps(world, 1_000_000, bench.SWEEPS, total / 10)}, f)


if __name__ == "__main__":
    main()
