"""Multi-rank host paths on the CPU (gloo, two ranks, launched as the driver launches the
bench: torch.distributed.run on 127.0.0.1): the bench's process group, barrier and
max-over-ranks timing, the serving router that splits one request stream over the GPUs'
servers and the report merged over the ranks, and the reference arm, which rank 0 alone runs
and prints. No GPU, no NCCL."""
import json
import os
import socket
import subprocess
import sys

import pytest

from phipict_b200.serve import merge_reports, percentile, route

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import multirank_worker as mw  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torchrun(args, nproc=2, timeout=300):
    env = dict(os.environ, PHIPICT_B200_DIST_BACKEND="gloo", CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", str(nproc),
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port())] + args
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout)


def test_route_covers_the_stream_and_balances_the_work():
    stream = mw.synthetic_stream(40)
    for world in (1, 2, 3, 8):
        shares = route(stream, world)
        rids = sorted(r.rid for s in shares for r in s)
        assert rids == list(range(40))
        loads = [sum(r.cost_hint for r in s) for s in shares]
        assert max(loads) - min(loads) <= max(r.cost_hint for r in stream)
        # deterministic: the same stream routes the same way on every rank
        assert [[r.rid for r in s] for s in route(stream, world)] == [[r.rid for r in s] for s in shares]
    # without estimates every request counts as one: round robin in arrival order
    plain = [mw.Request(rid=k, build=None, stuart=1.0, e_b=(0, 1, 0), steps=1, dt=1.0, arrival=float(k)) for k in range(6)]
    assert [[r.rid for r in s] for s in route(plain, 2)] == [[0, 2, 4], [1, 3, 5]]


def test_merged_report_takes_percentiles_over_all_requests():
    a = {"requests": 2, "failed": 0, "wall_s": 3.0, "batch_steps": 4, "peak_held_bytes": 5, "latencies": [1.0, 4.0],
         "cell_steps": 6_000_000, "cells_total": 60}
    b = dict(a, wall_s=2.0, latencies=[2.0, 3.0, 9.0], requests=3, failed=1, cell_steps=3_000_000)
    m = merge_reports([a, b])
    assert m["requests"] == 5 and m["failed"] == 1 and m["wall_s"] == 3.0
    assert m["latencies"] == [1.0, 2.0, 3.0, 4.0, 9.0]
    assert m["p50_s"] == percentile(m["latencies"], 50) == 3.0 and m["p99_s"] == 9.0
    assert m["mcell_steps_per_s"] == pytest.approx(9.0 / 3.0)


def test_two_gloo_ranks_plumbing_router_and_merged_report(tmp_path):
    res = _torchrun([os.path.join("tests", "multirank_worker.py"), str(tmp_path)])
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-4000:]
    outs = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in range(2)]
    stream = mw.synthetic_stream(23)
    shares = route(stream, 2)
    expect = merge_reports([mw.fake_report(shares[k], k) for k in range(2)])
    for k, o in enumerate(outs):
        assert o["rank"] == k and o["world"] == 2
        assert o["max"] == 2.5
        assert o["rids"] == [[r.rid for r in s] for s in shares]
        assert o["merged"] == json.loads(json.dumps(expect))


def test_reference_arm_prints_one_line_from_rank_zero():
    from oracle import build as ob

    ob.build()
    res = _torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"], timeout=900)
    assert res.returncode == 0, res.stderr[-4000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
