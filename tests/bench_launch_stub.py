"""A rank of bench.py's multi-rank plumbing on CPU (gloo): started by
bench.relaunch the way `bench.py --gpus N` starts its ranks, it takes its
rank from the launcher's environment with bench.dist_setup, joins the group
with bench.init_group, times a rank-dependent amount of host work and
reduces the times with bench.max_over_ranks; each rank writes what it saw to
<out>/rank<r>.json.  Used by tests/test_bench_launch.py."""

import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--out", required=True)
    args = ap.parse_args()
    rank, world, local = bench.dist_setup(args)
    bench.init_group(world, "gloo", timeout_s=60)
    t0 = time.perf_counter()
    time.sleep(0.05 * (rank + 1))
    mine = (time.perf_counter() - t0) * 1e3
    worst = bench.max_over_ranks(mine, world, device="cpu")
    with open(os.path.join(args.out, "rank%d.json" % rank), "w") as f:
        json.dump({"rank": rank, "world": world, "local": local, "ms": mine, "max_ms": worst}, f)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
