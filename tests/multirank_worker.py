"""One rank of the multi-rank host checks (launched by tests/test_multirank.py under
torch.distributed.run with the gloo backend, no GPU): the bench's rank plumbing (process
group, barrier, max over ranks) and the serving router with the merged report. Writes its
findings to <outdir>/rank<k>.json."""
import json
import os
import sys
from types import SimpleNamespace

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import torch.distributed as dist  # noqa: E402

import bench  # noqa: E402
from phipict_b200.serve import Request, gather_reports, route  # noqa: E402


def synthetic_stream(n):
    """Requests with arrival times and work estimates only (nothing is built)."""
    return [Request(rid=k, build=lambda: None, stuart=1.0, e_b=(0.0, 1.0, 0.0), steps=10, dt=1e-3,
                    arrival=0.05 * k, cost_hint=float((k % 5 + 1) * 1000)) for k in range(n)]


def fake_report(reqs, rank):
    """The report a server would give for `reqs` (latency and work derived from the request)."""
    lat = sorted(1.0 + 0.1 * r.rid + rank for r in reqs)
    cell_steps = int(sum(r.cost_hint for r in reqs))
    return {"requests": len(reqs), "failed": 0, "p50_s": None, "p99_s": None, "wall_s": 2.0 + rank,
            "mcell_steps_per_s": None, "batch_steps": 10 * len(reqs), "peak_held_bytes": 100 * (rank + 1),
            "latencies": lat, "cell_steps": cell_steps, "cells_total": cell_steps // 10}


def main(outdir):
    rank, world, local = bench.dist_setup(SimpleNamespace(impl="ours"))
    assert dist.is_initialized() and dist.get_backend() == "gloo"
    bench.barrier(world)
    mx = bench.max_over_ranks(rank + 1.5, world)
    stream = synthetic_stream(23)
    shares = route(stream, world)
    mine = shares[rank]
    every: list = [None] * world
    dist.all_gather_object(every, [r.rid for r in mine])
    merged = gather_reports(fake_report(mine, rank), world)
    out = {"rank": rank, "world": world, "max": mx, "rids": every, "merged": merged}
    with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
        json.dump(out, f)
    bench.barrier(world)
    dist.destroy_process_group()


if __name__ == "__main__":
    main(sys.argv[1])
