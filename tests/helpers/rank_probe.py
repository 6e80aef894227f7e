"""Started by tests/test_bench_ranks.py through bench.spawn_ranks: joins a gloo group and
reports, per rank, the world size it saw and bench.max_over_ranks of (rank + 1)."""
import datetime
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import torch.distributed as dist  # noqa: E402

import bench  # noqa: E402

if __name__ == "__main__":
    out_dir = sys.argv[1]
    rank, world, _ = bench._dist()
    bench.check_world(int(sys.argv[2]), world)
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    m = bench.max_over_ranks(float(rank + 1), world, "cpu")
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"rank": rank, "world": world, "max": m}, f)
    dist.barrier()
    dist.destroy_process_group()
