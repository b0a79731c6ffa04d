"""Benchmark of the phipict_b200 PISO/MHD step (one JSON line on rank 0).

Workload (default ``duct3d``): the 3D MHD rectangular duct of 3 connected blocks of
64x48x48 cells (442,368 cells), tanh wall stretching beta=2 in y and z, Ha=100, Re=1000
(N = 10), inflow u=1 plus seeded 1e-2 noise with a flux-balancing outflow, insulating walls
and an open-potential outflow. Fields are float64; every solve runs float32 Krylov
iterations inside float64 iterative refinement to a relative residual of 1e-10.
Synthetic inputs (seeded), no dataset. A step is one PISO step (momentum predictor,
2 pressure correctors) plus the potential step and the Lorentz force. The pressure and
potential solves start from the Galerkin projection of their solution onto the span of
their last 12 results, taken with the current matrix (``extrapolate_guesses``;
``--extrapolate-order`` for a polynomial extrapolation of fixed degree, ``adaptive`` or
another projection size;
``--no-extrapolate`` for phiPICT's zero pressure guess and previous potential); the plain
FP64 comparison leg keeps phiPICT's defaults.

``--impl reference`` times the CPU oracle (the restatement of phiPICT's step; phiPICT has no
CPU path) on the same workload with all host threads, on rank 0.

Multi-GPU: independent replicas (one instance per rank, no collective in the step);
``value`` counts the cells of all ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402
import torch  # noqa: E402

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "source": "fallback"}


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        d["source"] = "measured"
        return d
    return dict(PEAKS_FALLBACK)


def make_duct(device, dtype, nx=64, ny=48, nz=48, nblocks=3, seed=0):
    import phipict_b200 as pb
    from phipict_b200.grid import make_weights_tanh, rectilinear_vertices, span

    ys = span(-1.0, 1.0, make_weights_tanh(ny, 2.0))
    zs = span(-1.0, 1.0, make_weights_tanh(nz, 2.0))
    Re = 1000.0
    dom = pb.Domain(3, torch.tensor([1.0 / Re]), name="duct", device=device, dtype=dtype)
    blocks = []
    for i in range(nblocks):
        xs = np.linspace(2.0 * i, 2.0 * (i + 1), nx + 1)
        blocks.append(dom.CreateBlock(vertexCoordinates=rectilinear_vertices(xs, ys, zs, dtype=dtype), name=f"b{i}"))
    for i in range(nblocks - 1):
        blocks[i].ConnectBlock("+x", blocks[i + 1], "-x", "-y", "-z")
    g = torch.Generator(device="cpu").manual_seed(seed)
    inflow = torch.zeros(1, 3, nz, ny, 1, dtype=dtype)
    inflow[0, 0] = 1.0 + 1e-2 * torch.randn(nz, ny, 1, generator=g, dtype=dtype)
    blocks[0].CloseBoundary("-x", inflow.to(device))
    blocks[-1].CloseBoundary("+x", inflow.clone().to(device))
    blocks[-1].getBoundary("+x").setPotentialBC(pb.PotentialBC.OPEN)
    for b in blocks:
        for f in ("-y", "+y", "-z", "+z"):
            b.CloseBoundary(f)
    for b in blocks:
        v = torch.zeros(b.velocity.shape, dtype=dtype)
        v[:, 0] = 1.0
        v += 1e-2 * torch.randn(v.shape, generator=g, dtype=dtype)
        b.velocity.copy_(v.to(device))
    return dom


def make_hartmann2d(device, dtype, nx, ny, Re, seed=0, length=4.0):
    """Periodic 2D channel [0, length] x [-1, 1], no-slip insulating walls, u = 1 + 1e-3 noise."""
    import phipict_b200 as pb
    from phipict_b200.grid import rectilinear_vertices

    dom = pb.Domain(2, torch.tensor([1.0 / Re]), name="hartmann", device=device, dtype=dtype)
    b = dom.CreateBlock(vertexCoordinates=rectilinear_vertices(np.linspace(0.0, length, nx + 1),
                                                               np.linspace(-1.0, 1.0, ny + 1), dtype=dtype), name="channel")
    b.CloseBoundary("-y")
    b.CloseBoundary("+y")
    b.MakePeriodic("x")
    g = torch.Generator(device="cpu").manual_seed(seed)
    v = torch.zeros(b.velocity.shape, dtype=dtype)
    v[:, 0] = 1.0
    v += 1e-3 * torch.randn(v.shape, generator=g, dtype=dtype)
    b.velocity.copy_(v.to(device))
    return dom


def make_cavity2d(device, dtype, n, Re, seed=0):
    """Lid-driven cavity [0, 1]^2 from rest: four no-slip insulating walls, the +y lid at u = 1."""
    import phipict_b200 as pb
    from phipict_b200.grid import rectilinear_vertices

    dom = pb.Domain(2, torch.tensor([1.0 / Re]), name="cavity", device=device, dtype=dtype)
    xs = np.linspace(0.0, 1.0, n + 1)
    b = dom.CreateBlock(vertexCoordinates=rectilinear_vertices(xs, xs, dtype=dtype), name="cavity")
    for f in ("-x", "+x", "-y"):
        b.CloseBoundary(f)
    lid = torch.zeros(1, 2, 1, n, dtype=dtype)
    lid[0, 0] = 1.0
    b.CloseBoundary("+y", lid.to(device))
    g = torch.Generator(device="cpu").manual_seed(seed)
    b.velocity.copy_((1e-3 * torch.randn(b.velocity.shape, generator=g, dtype=dtype)).to(device))
    return dom


WORKLOADS = {
    "duct3d": dict(nx=64, ny=48, nz=48, nblocks=3, Ha=100.0, Re=1000.0, dt=0.01, rtol=1e-10),
    # 64 heterogeneous 2D instances (Hartmann channels and lid-driven cavities) in one batch
    "batch64": dict(instances=64, sides=(32, 48, 64, 96, 128, 192, 256), rtol=1e-8),
    # a served Poisson stream of 2D and 3D requests
    "serve": dict(requests=24, rate=20.0, steps=100, rtol=1e-8),
    # differentiable duct: 96^3 cells in 2 blocks, 50 steps with checkpoints every 10
    "adjoint": dict(nx=48, ny=96, nz=96, nblocks=2, Ha=10.0, Re=1000.0, dt=0.01, rollout=50, every=10, rtol=1e-12),
    # every kernel on single-block grids far larger than L2 (SWEEP_GRIDS)
    "sweep": dict(),
}


def algorithmic_cg_bytes(dims: int, s_A: int, s_v: int) -> int:
    """Bytes per cell of one fused CG iteration (kCgDirection + kCgUpdate): the stencil
    (2d+1 values, no indices) and 10 vector passes (r, p_in read / p_out, q written; x, p, r,
    q read / x, r written)."""
    return (2 * dims + 1) * s_A + 10 * s_v


def algorithmic_pcg_bytes(dims: int, levels: list[int], dense_doubles: int = 0) -> float:
    """Bytes per fine cell of one multigrid-preconditioned float32 CG iteration: the CG
    passes (algorithmic_cg_bytes with z in place of r in the direction) plus, per cycle level
    l of n_l cells, the restriction (stencil + b read, coarse b written) and the prolongation
    with its smoothing sweep (stencil, b and the coarse correction read, z written), plus the
    dense operator of the last cycle level (dense_doubles FP64 values)."""
    st = (2 * dims + 1) * 4
    cyc = 0.0
    for l in range(len(levels) - 1):
        frac = levels[l] / levels[0]
        coarse = levels[l + 1] / levels[0]
        cyc += frac * (st + 4) + coarse * 4          # restriction
        cyc += frac * (st + 4 + 4) + coarse * 4      # prolongation + post-smoothing
    return algorithmic_cg_bytes(dims, 4, 4) + cyc + 8.0 * dense_doubles / levels[0]


# DRAM bytes per preconditioned CG iteration on the duct workload, from a full ncu capture of
# one persistent launch (the first inner solve of the timed step: 26.11 MB read + 0.57 MB
# written in a 24-iteration solve): the working set is L2-resident
PCG_DRAM_BYTES_PER_ITERATION_DUCT3D = (26.11e6 + 0.57e6) / 24


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"phb_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), smmax=float(parts[2]), power=float(parts[3]), hw=parts[5],
                                 hwt=parts[6], swt=parts[7], swp=parts[8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        reasons = []
        for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"), ("swt", "sw_thermal_slowdown"),
                          ("swp", "sw_power_cap")):
            if any(r[key].lower() == "active" for r in rows):
                reasons.append(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in rows), "sm_max_mhz": max(r["smmax"] for r in rows),
                "power_w_max": max(r["power"] for r in rows), "samples": len(rows), "reasons": reasons}


def dist_setup(args):
    """Rank, world size and local rank from the torchrun environment. With more than one rank a
    process group is formed (NCCL on GPUs; gloo without CUDA, or when PHIPICT_B200_DIST_BACKEND
    says so). The reference arm forms none: rank 0 alone runs it, the others leave at once."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if torch.cuda.is_available():
        torch.cuda.set_device(local if world > 1 else 0)
    if world > 1 and args.impl != "reference":
        import datetime

        import torch.distributed as dist

        backend = os.environ.get("PHIPICT_B200_DIST_BACKEND") or ("nccl" if torch.cuda.is_available() else "gloo")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def max_over_ranks(v: float, world: int) -> float:
    """The largest of every rank's v (the device times of a step loop)."""
    if world == 1:
        return v
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def extrapolate_order(v: str):
    return v if v == "adaptive" or v.startswith("projection") else int(v)


def guess_label(order) -> str:
    if isinstance(order, str) and order.startswith("projection"):
        n = int(order.split(":", 1)[1]) if ":" in order else 12
        return f"Galerkin projection onto the span of the last {n} results"
    if order == "adaptive":
        return ("extrapolated from the last results, the degree (<= 4) that predicted the previous "
                "result best")
    return f"degree-{order} polynomial extrapolation from the last {order + 1} results"


def build_sim(wl: dict, device, mixed: bool, amg: bool = True, warm: bool = False, autotune: bool = False,
              extrapolate: int | str = 0):
    import phipict_b200 as pb

    dtype = torch.float64
    dom = make_duct(device, dtype, wl["nx"], wl["ny"], wl["nz"], wl["nblocks"])
    dom.PrepareSolve()
    N = wl["Ha"] ** 2 / wl["Re"]
    tol = pb.SolverTolerance(rtol=wl["rtol"])

    def reset_source(domain, **kw):
        # the Lorentz force is added onto the velocity source (simulation/mhd.py:583-593);
        # the benchmark resets it each step, as phiPICT's examples/hartmann.py does
        for b in domain.getBlocks():
            if b.velocitySource is not None:
                b.velocitySource.zero_()

    hooks = pb.Hooks().append(pb.Hook.PRE_VELOCITY_SETUP, reset_source)
    sim = pb.MHDSimulation(dom, wl["dt"], torch.tensor(N), torch.tensor([0.0, 1.0, 0.0], dtype=dtype),
                           non_orthogonal=False, advection_tol=tol, pressure_tol=tol, potential_tol=tol,
                           mixed_precision=mixed, hooks=hooks, pressure_use_amg=amg and mixed,
                           potential_use_preconditioner=amg and mixed, pressure_warm_start=warm,
                           autotune_solvers=autotune, extrapolate_guesses=extrapolate)
    return dom, sim


def run_ours(args, rank, world, local):
    wl = WORKLOADS[args.workload]
    device = torch.device("cuda", local)
    mixed = not args.plain_fp64
    amg = mixed and not args.no_amg
    dom, sim = build_sim(wl, device, mixed, amg, args.pressure_warm_start, args.autotune,
                         args.extrapolate_order if args.extrapolate and mixed else 0)
    if args.inner_rtol:
        sim.refinement_inner_rtol = args.inner_rtol
    cells = dom.getTotalSize()
    stream = torch.cuda.current_stream(device)
    for _ in range(tuned_warmup(args, sim)):
        if not sim.single_step():
            raise RuntimeError("warm-up step failed")
    torch.cuda.synchronize()
    # solve timing: CUDA events around each solve graph launch (on the launching stream)
    sim._solve_events = []
    infos = []
    orig_collect = sim.collect_solves

    def collect(raise_on_failure=True):
        ok = orig_collect(raise_on_failure)
        infos.extend(sim.solve_report())
        return ok

    sim.collect_solves = collect
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        if not sim.single_step():
            raise RuntimeError("timed step failed")
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = t0.elapsed_time(t1)
    ms = max_over_ranks(ms, world)
    final = (dom._u_block.clone(), dom.pressureResult.clone(), dom.epotResult.clone())
    # solver statistics of the timed steps
    solve_ms = 0.0
    per_tag: dict = {}
    for a, b, tag in sim._solve_events:
        t = a.elapsed_time(b)
        solve_ms += t
        per_tag[tag] = per_tag.get(tag, 0.0) + t / args.steps
    tag_its: dict = {}
    for tag, lst in infos:
        tag_its[tag] = tag_its.get(tag, 0) + sum(i.innerIterations if mixed else i.usedIterations for i in lst) / args.steps
    inner_its = sum(i.innerIterations if mixed else i.usedIterations for _, lst in infos for i in lst)
    sweeps = sum(i.usedIterations for _, lst in infos for i in lst) if mixed else 0
    sim._solve_events = None
    # end-to-end: the same trajectory as the timed steps (a second simulation built and warmed
    # up the same way), every step reading its velocity from pinned host memory and writing u,
    # p and phi back there; the next step starts from the velocity it wrote
    d = dom.getSpatialDims()
    dom_e, sim_e = build_sim(wl, device, mixed, amg, args.pressure_warm_start, args.autotune,
                             args.extrapolate_order if args.extrapolate and mixed else 0)
    if args.inner_rtol:
        sim_e.refinement_inner_rtol = args.inner_rtol
    for _ in range(tuned_warmup(args, sim_e)):
        if not sim_e.single_step():
            raise RuntimeError("warm-up step failed")
    nu = dom_e._u_block.numel()
    h_out = torch.empty(nu + 2 * cells, dtype=dom_e.getDtype(), pin_memory=True)
    h_out[:nu].copy_(dom_e._u_block.view(-1))
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e_steps = args.steps
    e0.record(stream)
    for _ in range(e_steps):
        dom_e._u_block.view(-1).copy_(h_out[:nu], non_blocking=True)
        if not sim_e.single_step():
            raise RuntimeError("end-to-end step failed")
        h_out[:nu].copy_(dom_e._u_block.view(-1), non_blocking=True)
        h_out[nu:nu + cells].copy_(dom_e.pressureResult, non_blocking=True)
        h_out[nu + cells:].copy_(dom_e.epotResult, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world) / e_steps
    del sim_e, dom_e
    plain = (plain_fp64_leg(args, wl, device, stream, final, world, tuned_warmup(args, sim))
             if (mixed and not args.no_fp64_leg) else None)
    total_cells = cells * world
    value = total_cells * args.steps / (ms / 1e3) / 1e6
    if plain:
        plain["vs_plain_fp64"]["mixed_over_plain"] = round(value / plain["vs_plain_fp64"]["value"], 3)
    # roofline of the dominant kernel: the (preconditioned) Krylov iteration, float32 when
    # mixed; solve time / inner iterations. The momentum BiCGStab iterations (about a tenth of
    # the iterations) are charged at the PCG's bytes per cell, which undercounts them (a 3-RHS
    # float32 BiCGStab iteration moves 2(2d+1)*4 + 18d*4 = 272 B/cell in 3D): the achieved
    # figure is conservative
    s = 4 if mixed else 8
    hier = sim._amg_cache.get("P") if amg else None
    levels = hier.sizes if hier is not None else None
    if hier is not None:
        cycle = hier.sizes[:hier.tail_level + 1]
        per_cell = algorithmic_pcg_bytes(d, cycle, hier.coarse_inv.numel())
    else:
        per_cell = algorithmic_cg_bytes(d, s, s)
    it_time_ms = solve_ms / max(1, inner_its)
    achieved = per_cell * cells / (it_time_ms / 1e3) / 1e9 if inner_its else None
    pk = peaks()
    # launches: assembly, mean projections and copies per PISO+MHD step; per solve kInit(Outer)
    # and per refinement sweep kRefineResidual, kInit, the persistent solve and kRefineUpdate;
    # per step the pressure hierarchy's setup (Galerkin per level, dense, inverse)
    launches_per_step = 26
    setup = (2 * len(levels) + 6) if levels else 0
    gpu_launches = args.steps * (launches_per_step + setup) + 4 * max(1, sweeps) + len(infos)
    return dict(
        metric="Mcell-steps/s", value=round(value, 4), unit="Mcell-steps/s", n_gpus=world, steps=args.steps,
        warmup=args.warmup, ms_per_step=round(ms / args.steps, 4), higher_is_better=True, scaling="weak",
        vs_baseline=None, dtype="f64 fields, f32 Krylov + f64 refinement" if mixed else "f64",
        data="synthetic (seeded inflow noise 1e-2, seeded initial state)",
        config={"workload": f"{args.workload}: 3 blocks 64x48x48 (442,368 cells), Ha=100, Re=1000, dt=0.01, "
                            f"rtol 1e-10, {'mixed precision' if mixed else 'plain fp64'}"
                            f"{', multigrid-preconditioned pressure and potential CG' if amg else ''}",
                "amg_levels": levels,
                "amg_refresh": ("full pressure multigrid setup on every 4th matrix change, the finest level "
                                "in between (coarse_refresh_interval 4)") if amg else None,
                "initial_guesses": (guess_label(args.extrapolate_order) if args.extrapolate and mixed else
                                    "previous step's pressure" if args.pressure_warm_start else
                                    "zero pressure, previous step's potential"),
                "cells_per_gpu": cells, "l2": "working set ~60 MB f32 fits L2; HBM claims on the roofline sweep",
                "parallelism": f"replicas x{world}"},
        clocks=clk,
        e2e={"value": round(total_cells / (e2e_ms / 1e3) / 1e6, 4), "unit": "Mcell-steps/s",
             "h2d_bytes_per_step": int(nu * h_out.element_size()),
             "d2h_bytes_per_step": int(h_out.numel() * h_out.element_size())},
        roofline={"bound": "hbm",
                  "limited_by": ("grid-barrier and L2 latency: the ~60 MB working set stays in L2 (DRAM traffic "
                                 "is ~1.5 % of the algorithmic bytes), so the fraction of HBM peak is low by "
                                 "construction; HBM-bound fractions are measured by the roofline sweep") if amg else None,
                  "kernel": ("persistent PCG iteration (V-cycle + direction + update, kCgPersistent)" if amg
                             else "CG iteration (kCgDirection + kCgUpdate)"),
                  "achieved": round(achieved, 1) if achieved else None, "peak": pk.get("hbm_gbs"),
                  "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 4) if achieved else None,
                  "traffic": (round(PCG_DRAM_BYTES_PER_ITERATION_DUCT3D) if hier is not None and args.workload == "duct3d"
                              else None),
                  "traffic_unit": "DRAM bytes per iteration (ncu capture)",
                  "algorithmic_bytes_per_iteration": round(per_cell * cells),
                  "bytes_per_cell": round(per_cell, 2), "peak_source": pk["source"],
                  "iterations": inner_its, "solve_ms": round(solve_ms, 3)},
        gpu_launches=int(gpu_launches),
        **({"solver_tuning": sim.solver_tuner.report()} if sim.solver_tuner is not None else {}),
        **({"vs_plain_fp64": plain["vs_plain_fp64"], "err_vs_fp64": plain["err_vs_fp64"]} if plain else {}),
        solver={"inner_iterations_per_step": round(inner_its / args.steps, 1),
                "refinement_sweeps_per_step": round(sweeps / args.steps, 2),
                "ms_per_step_by_solve": {k: round(v, 3) for k, v in per_tag.items()},
                "iterations_per_step_by_solve": {k: round(v, 1) for k, v in tag_its.items()}},
    )


def plain_fp64_leg(args, wl, device, stream, final, world, warmup: int) -> dict:
    """The plain FP64 single-instance path (FP64 CG / BiCGStab, no refinement, no multigrid) on
    the same workload: the same warm-up and timed step counts from the same initial state, timed
    with CUDA events; its fields after the same number of steps are the all-FP64 run that the
    mixed-precision fields are compared with (relative L2 error per field). Its initial guesses
    are phiPICT's defaults (zero pressure, the previous potential)."""
    dom, sim = build_sim(wl, device, False, False)
    for _ in range(warmup):
        if not sim.single_step():
            raise RuntimeError("plain FP64 warm-up step failed")
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        if not sim.single_step():
            raise RuntimeError("plain FP64 step failed")
    b.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(a.elapsed_time(b), world) / args.steps
    cells = dom.getTotalSize() * world
    ref = (dom._u_block, dom.pressureResult, dom.epotResult)

    def rel(x, y):
        return float(torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y))

    err = {k: rel(x, y) for k, x, y in zip(("u", "p", "phi"), final, ref)}
    value = cells / (ms / 1e3) / 1e6
    return {"vs_plain_fp64": {"value": round(value, 4), "unit": "Mcell-steps/s", "ms_per_step": round(ms, 3),
                              "dtype": "f64", "path": "FP64 CG pressure/potential, FP64 BiCGStab momentum, no refinement, "
                                                      "no multigrid, one instance",
                              "steps": args.steps, "warmup": warmup},
            "err_vs_fp64": {**{k: float(f"{v:.3e}") for k, v in err.items()},
                            "norm": "relative L2 against the plain FP64 run after the same warm-up + timed steps"}}


def cpu_baseline(wl, sample_steps=1, min_seconds=0.0, max_steps=8) -> dict:
    """The oracle's FP64 step on the host cores (bounded sample): sample_steps steps, then more
    while the sample is shorter than min_seconds (at most max_steps in all)."""
    from oracle.oracle import OracleDomain, OracleSim
    import phipict_b200 as pb

    dom = make_duct("cpu", torch.float64, wl["nx"], wl["ny"], wl["nz"], wl["nblocks"])
    od = OracleDomain(dom)
    u0 = np.concatenate([b.velocity.reshape(3, -1).numpy() for b in dom.getBlocks()], axis=1).reshape(-1)
    tol = pb.SolverTolerance(rtol=wl["rtol"])
    N = wl["Ha"] ** 2 / wl["Re"]
    sim = OracleSim(od, u0, wl["dt"], 1.0 / wl["Re"], advection_tol=tol, pressure_tol=tol,
                    mhd=dict(stuart=N, e_b=[0.0, 1.0, 0.0], singular=True, potential_tol=tol))
    t = time.perf_counter()
    done = 0
    while done < sample_steps or (time.perf_counter() - t < min_seconds and done < max_steps):
        sim.src = None
        sim.step()
        done += 1
    el = time.perf_counter() - t
    sample_steps = done
    return {"value": round(od.n * sample_steps / el / 1e6, 5), "unit": "Mcell-steps/s",
            "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)), "kind": "port",
            "sample": f"{sample_steps} oracle PISO+MHD step(s) of the {od.n}-cell duct, float64, {el:.1f} s",
            "seconds": round(el, 2)}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    wl = WORKLOADS[args.workload]
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    for _ in range(args.warmup):
        pass  # the oracle has no warm-up state; its first step is representative
    steps = max(1, args.steps if args.steps <= 2 else 2)
    base = cpu_baseline(wl, steps)
    line = dict(metric="Mcell-steps/s", value=base["value"], unit="Mcell-steps/s", n_gpus=world, steps=steps,
                warmup=args.warmup, ms_per_step=round(base["seconds"] * 1e3 / steps, 1), higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype="f64", data="synthetic", impl="reference",
                config={"workload": f"{args.workload}: 3 blocks 64x48x48 (442,368 cells), Ha=100, Re=1000",
                        "parallelism": "host cores"},
                cpu_baseline=base,
                e2e={"value": base["value"], "unit": "Mcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    return line


def batch64_instances(wl, device, dtype, seed=0):
    """The seeded instance mix: (domain, stuart, dt) per instance; sides uniform over
    wl['sides'], Hartmann channel or cavity by a fair coin, Ha log-uniform in [1, 1000],
    Re uniform in [100, 2000]; dt = min(1e-3, 0.5 / N) keeps the explicit Lorentz force stable."""
    g = torch.Generator().manual_seed(seed)
    out = []
    for k in range(wl["instances"]):
        side = wl["sides"][int(torch.randint(len(wl["sides"]), (1,), generator=g))]
        cavity = bool(torch.rand(1, generator=g) < 0.5)
        Ha = float(10 ** (3 * torch.rand(1, generator=g)))
        Re = float(100 + 1900 * torch.rand(1, generator=g))
        dom = make_cavity2d(device, dtype, side, Re, seed=k) if cavity else make_hartmann2d(device, dtype, side, side, Re, seed=k)
        dom.PrepareSolve()
        N = Ha * Ha / Re
        out.append((dom, N, min(1e-3, 0.5 / N)))
    return out


def reset_cell_source(domain, **kw):
    """The Lorentz force is added onto the velocity source (simulation/mhd.py:583-593); the
    benchmarks reset the source every step, as phiPICT's examples/hartmann.py does."""
    if getattr(domain, "_src", None) is not None:
        domain._src.zero_()


def tuned_warmup(args, sim) -> int:
    """Warm-up steps: with --autotune at least enough for every solve's tuning trials."""
    t = sim.solver_tuner
    return args.warmup if t is None else max(args.warmup, t.trials * len(t.CANDIDATES) + 1)


def run_batch64(args, rank, world, local):
    import phipict_b200 as pb

    wl = WORKLOADS["batch64"]
    device = torch.device("cuda", local)
    inst = batch64_instances(wl, device, torch.float64, seed=rank)
    cells = sum(d.numCells() for d, _, _ in inst)
    batch = pb.DomainBatch([d for d, _, _ in inst])
    tol = pb.SolverTolerance(rtol=wl["rtol"])
    sim = pb.MHDSimulation(batch, inst[0][2], torch.tensor([n for _, n, _ in inst], dtype=torch.float64),
                           torch.tensor([0.0, 1.0, 0.0], dtype=torch.float64), non_orthogonal=False,
                           advection_tol=tol, pressure_tol=tol, potential_tol=tol, mixed_precision=not args.plain_fp64,
                           pressure_use_amg=not args.plain_fp64 and not args.no_amg,
                           potential_use_preconditioner=not args.plain_fp64 and not args.no_amg,
                           hooks=pb.Hooks().append(pb.Hook.PRE_VELOCITY_SETUP, reset_cell_source),
                           autotune_solvers=args.autotune)
    sim.time_step = torch.tensor([dt for _, _, dt in inst], dtype=torch.float64)
    stream = torch.cuda.current_stream(device)
    for _ in range(tuned_warmup(args, sim)):
        if not sim.single_step():
            raise RuntimeError(f"warm-up step failed: {sim.last_error}")
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        if not sim.single_step():
            raise RuntimeError(f"timed step failed: {sim.last_error}")
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(t0.elapsed_time(t1), world)
    # the same instances one at a time (plain FP64 path, one timed step each after a warm-up)
    alone_ms = 0.0
    if not args.no_alone:
        for dom, N, dt in batch64_instances(wl, device, torch.float64, seed=rank):
            s1 = pb.MHDSimulation(dom, dt, torch.tensor([N], dtype=torch.float64),
                                  torch.tensor([0.0, 1.0, 0.0], dtype=torch.float64), non_orthogonal=False,
                                  advection_tol=tol, pressure_tol=tol, potential_tol=tol,
                                  hooks=pb.Hooks().append(pb.Hook.PRE_VELOCITY_SETUP, reset_cell_source))
            s1.single_step()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            s1.single_step()
            b.record(stream)
            torch.cuda.synchronize()
            alone_ms += a.elapsed_time(b)
    value = cells * world * args.steps / (ms / 1e3) / 1e6
    return dict(metric="Mcell-steps/s", value=round(value, 4), unit="Mcell-steps/s", n_gpus=world, steps=args.steps,
                warmup=tuned_warmup(args, sim), ms_per_step=round(ms / args.steps, 4), higher_is_better=True,
                scaling="weak", vs_baseline=None,
                dtype="f64 fields, f32 Krylov + f64 refinement" if not args.plain_fp64 else "f64",
                data="synthetic (seeded instance mix)",
                config={"workload": f"batch64: {len(inst)} 2D Hartmann/cavity instances, sides in {wl['sides']}, "
                                    f"Ha log-uniform [1,1000], Re U(100,2000), one DomainBatch, rtol {wl['rtol']}",
                        "cells_per_gpu": cells, "parallelism": f"replicas x{world}"},
                clocks=clk,
                **({"solver_tuning": sim.solver_tuner.report()} if sim.solver_tuner is not None else {}),
                one_at_a_time={"ms_per_step": round(alone_ms, 3) if alone_ms else None,
                               "value": round(cells / (alone_ms / 1e3) / 1e6, 4) if alone_ms else None,
                               "path": "plain FP64, each instance alone"},
                gpu_launches=None)


def batch64_record(args, rank, world, local) -> dict:
    """A compact run of the heterogeneous batch (64 2D instances in one DomainBatch, 2 warm-up
    and 5 timed steps) with the same instances stepped one at a time on the plain FP64 path:
    the batched, mixed-precision path against the plain single-instance path, both timed with
    CUDA events in this run."""
    sub = argparse.Namespace(**vars(args))
    sub.steps, sub.warmup, sub.plain_fp64, sub.no_alone = 5, 2, False, False
    r = run_batch64(sub, rank, world, local)
    alone = r["one_at_a_time"]["value"]
    return {"workload": r["config"]["workload"], "cells": r["config"]["cells_per_gpu"], "value": r["value"],
            "unit": "Mcell-steps/s", "ms_per_step": r["ms_per_step"], "steps": sub.steps, "warmup": sub.warmup,
            "dtype": r["dtype"], "one_at_a_time": r["one_at_a_time"],
            "batched_over_one_at_a_time": round(r["value"] / alone, 2) if alone else None}


def serve_requests(wl, device, seed=0):
    """The seeded request stream: half 2D Hartmann channels with side U[64, 512], half 3D
    ducts of one block with side U[32, 128]; Ha log-uniform in [1, 1000], Re = 1000."""
    from phipict_b200.serve import Request, poisson_arrivals

    g = torch.Generator().manual_seed(seed)
    arrivals = poisson_arrivals(wl["requests"], wl["rate"], seed)
    reqs = []
    for k in range(wl["requests"]):
        three = bool(torch.rand(1, generator=g) < 0.5)
        side = int(32 + 96 * torch.rand(1, generator=g)) if three else int(64 + 448 * torch.rand(1, generator=g))
        Ha = float(10 ** (3 * torch.rand(1, generator=g)))
        N = Ha * Ha / 1000.0
        dt = min(0.01 if three else 1e-3, 0.5 / N)

        def build(k=k, three=three, side=side):
            dom = (make_duct(device, torch.float64, side, side, side, 1, seed=k) if three
                   else make_hartmann2d(device, torch.float64, side, side, 1000.0, seed=k))
            dom.PrepareSolve()
            return dom
        reqs.append(Request(rid=k, build=build, stuart=N, e_b=(0.0, 1.0, 0.0), steps=wl["steps"], dt=dt,
                            arrival=arrivals[k], cost_hint=float(side ** (3 if three else 2) * wl["steps"])))
    return reqs


def serve_one_at_a_time(wl, device, tol, sample: int, steps: int) -> dict:
    """The first `sample` requests of the stream run one at a time on the plain FP64 path
    (FP64 CG/BiCGStab, no refinement, no multigrid), `steps` timed steps each after one
    warm-up step, CUDA events around each request's steps: its Mcell-steps/s."""
    import phipict_b200 as pb

    cell_steps, ms = 0, 0.0
    stream = torch.cuda.current_stream(device)
    reqs = serve_requests(dict(wl, requests=max(sample, 1)), device, seed=0)[:sample]
    for r in reqs:
        dom = r.build()
        sim = pb.MHDSimulation(dom, r.dt, torch.tensor([r.stuart], dtype=torch.float64),
                               torch.tensor(r.e_b, dtype=torch.float64), non_orthogonal=False, advection_tol=tol,
                               pressure_tol=tol, potential_tol=tol,
                               hooks=pb.Hooks().append(pb.Hook.PRE_VELOCITY_SETUP, reset_cell_source))
        sim.single_step()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            sim.single_step()
        b.record(stream)
        torch.cuda.synchronize()
        ms += a.elapsed_time(b)
        cell_steps += dom.numCells() * steps
        del sim, dom
    return {"value": round(cell_steps / (ms / 1e3) / 1e6, 4) if ms else None, "unit": "Mcell-steps/s",
            "sample": f"the first {sample} requests of the stream, {steps} steps each after one warm-up step, plain FP64"}


def run_serve(args, rank, world, local):
    import phipict_b200 as pb
    from phipict_b200.serve import Server, gather_reports, route

    wl = dict(WORKLOADS["serve"])
    if args.requests:
        wl["requests"] = args.requests
    device = torch.device("cuda", local)
    tol = pb.SolverTolerance(rtol=wl["rtol"])
    kw = dict(non_orthogonal=False, advection_tol=tol, pressure_tol=tol, potential_tol=tol,
              mixed_precision=not args.plain_fp64, pressure_use_amg=not args.plain_fp64,
              potential_use_preconditioner=not args.plain_fp64,
              hooks=pb.Hooks().append(pb.Hook.PRE_VELOCITY_SETUP, reset_cell_source))
    server = Server(device=device, hbm_budget=150e9, sim_kwargs=kw)
    # one stream of world x requests at world x the rate; every rank routes it the same way
    # and serves its share (weak scaling), the reports are merged over the ranks
    stream = serve_requests(dict(wl, requests=wl["requests"] * world, rate=wl["rate"] * world), device, seed=0)
    mine = route(stream, world)[rank]
    server.run(mine)
    rep = gather_reports(server.report(), world)
    cells = rep["cells_total"]
    plain = serve_one_at_a_time(wl, device, tol, args.plain_sample, args.plain_steps) if args.plain_sample else None
    return dict(metric="Mcell-steps/s", value=round(rep["mcell_steps_per_s"], 4), unit="Mcell-steps/s",
                n_gpus=world, steps=wl["steps"], warmup=0, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f64 fields, f32 Krylov + f64 refinement" if not args.plain_fp64 else "f64",
                data="synthetic (seeded Poisson request stream)",
                config={"workload": f"serve: {wl['requests']} requests at {wl['rate']}/s, 50% 2D side U[64,512], "
                                    f"50% 3D side U[32,128], Ha log-uniform [1,1000], {wl['steps']} steps each, "
                                    f"rtol {wl['rtol']}, admission against 150 GB", "parallelism": f"replicas x{world}"},
                served={"requests": rep["requests"], "p50_s": rep["p50_s"], "p99_s": rep["p99_s"],
                        "wall_s": round(rep["wall_s"], 3), "failed": rep["failed"], "batch_steps": rep["batch_steps"],
                        "joins_while_running": rep.get("joins"), "batch_rebuilds": rep.get("repacks"),
                        "cells_total": cells, "one_at_a_time_fp64": plain,
                        "failures": [f"{r.rid}: {r.failed[:160]}" for r in server.finished if r.failed][:4],
                        "peak_held_bytes": rep["peak_held_bytes"]},
                gpu_launches=None)


SWEEP_GRIDS = [(3, 128), (3, 192), (3, 256), (2, 2048), (2, 4096)]


def make_box(device, dims, n, Re=1000.0, seed=0, shear=0.0):
    """One block of n^dims cells on [0, 2] x [-1, 1]^(dims-1): periodic in x, no-slip
    insulating walls elsewhere, u = (1, 0, 0) plus seeded 1e-2 noise. shear > 0 shears the
    vertices, x += shear * y (a curvilinear grid with metric cross terms everywhere)."""
    import phipict_b200 as pb
    from phipict_b200.grid import rectilinear_vertices

    dtype = torch.float64
    dom = pb.Domain(dims, torch.tensor([1.0 / Re]), name="box", device=device, dtype=dtype)
    xs = np.linspace(0.0, 2.0, n + 1)
    ys = np.linspace(-1.0, 1.0, n + 1)
    v = rectilinear_vertices(xs, ys, *([ys] if dims == 3 else []), dtype=dtype)
    if shear:
        v[0, 0] = v[0, 0] + shear * v[0, 1]
    b = dom.CreateBlock(vertexCoordinates=v, name="box")
    for f in ("-y", "+y") + (("-z", "+z") if dims == 3 else ()):
        b.CloseBoundary(f)
    b.MakePeriodic("x")
    g = torch.Generator(device="cpu").manual_seed(seed)
    v = torch.zeros(b.velocity.shape, dtype=dtype)
    v[:, 0] = 1.0
    v += 1e-2 * torch.randn(v.shape, generator=g, dtype=dtype)
    b.velocity.copy_(v.to(device))
    return dom


def assembly_bytes(d: int, s: int = 8) -> dict:
    """Algorithmic bytes per cell of the assembly kernels (float64 fields, s bytes a value):
    every input and output once, per-cell transforms of 2d^2+1 values, stencils of 2d+1
    values without indices; the matrix kernels also write the float32 copy the inner solves
    use ((2d+1)*4 bytes)."""
    return {"advection_matrix": (d + 2 * d * d + 1 + 2 * d + 1 + 1) * s + (2 * d + 1) * 4,
            "advection_rhs": (3 * d + 1) * s,
            "pressure_matrix": (1 + d * d + 1 + 2 * d + 1) * s + (2 * d + 1) * 4,
            "pressure_rhs": (2 * d + 1 + 4 * d + 2) * s,
            "divergence": (d + d * d + 1 + 1) * s,
            "correct_velocity": (3 + d * d + 1 + 2 * d) * s,
            "uxb_epot_rhs": (d + 3) * s + (d + d * d + 1 + 1) * s,
            "current_lorentz": (1 + 3 + 2 * d * d + 1 + 3) * s + (3 + 2 * d) * s}


def run_sweep(args, rank, world, local):
    """Roofline sweep: every kernel of the step on single-block grids far larger than L2
    (128^3 ... 256^3, 2048^2, 4096^2), each launch timed alone with CUDA events after an L2
    flush; achieved = algorithmic bytes / time, frac = achieved / measured HBM peak. The
    Krylov iterations run a fixed iteration count (float32, as inside the refinement)."""
    import ctypes as ct

    import phipict_b200 as pb
    from phipict_b200 import _C as backend
    from phipict_b200 import _lib
    from phipict_b200.solvers import BICGSTAB, CG, MODES, solver_for

    device = torch.device("cuda", local)
    pk = peaks()
    peak = pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])
    grids = SWEEP_GRIDS if not args.sweep_grids else [tuple(int(v) for v in g.split("x")) for g in args.sweep_grids.split(",")]
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=device)
    reps = args.steps
    rows = []
    clocks = ClockSampler(local)
    clocks.start()
    for dims, n in grids:
        dom = make_box(device, dims, n, shear=args.sweep_shear)
        dom.PrepareSolve()
        tol = pb.SolverTolerance(rtol=1e-6)
        sim = pb.MHDSimulation(dom, 1e-3, torch.tensor(10.0), torch.tensor([0.0, 1.0, 0.0], dtype=torch.float64),
                               non_orthogonal=False, advection_tol=tol, pressure_tol=tol, potential_tol=tol,
                               mixed_precision=True, pressure_use_amg=True, potential_use_preconditioner=True)
        for _ in range(max(1, args.warmup)):
            if not sim.single_step():
                raise RuntimeError(f"warm-up step failed on {n}^{dims}: {sim.last_error}")
        cells = dom.numCells()
        S = _lib.stream_ptr(device)
        ts = sim._time_step_tensor(None)
        desc = dom.desc()
        kern = {
            "advection_matrix": lambda: backend.SetupAdvectionMatrix(dom, ts, 0),
            "advection_rhs": lambda: backend.SetupAdvectionVelocity(dom, ts, 0, False),
            "pressure_matrix": lambda: backend.SetupPressureMatrix(dom, ts, 0, False),
            "pressure_rhs": lambda: _lib.call("phb_pressure_rhs", ct.byref(desc), dom._C_st.data_ptr(), dom.A.data_ptr(),
                                              dom._u_block.data_ptr(), dom.velocityResult.data_ptr(), *backend._src(dom),
                                              dom.pressureRHS.data_ptr(), S),
            "divergence": lambda: _lib.call("phb_divergence", ct.byref(desc), dom.pressureRHS.data_ptr(),
                                            dom.pressureRHSdiv.data_ptr(), S),
            "correct_velocity": lambda: backend.CorrectVelocity(dom, ts, version=1),
            "uxb_epot_rhs": lambda: _lib.call("phb_uxb_epot_rhs", ct.byref(desc), dom.velocityResult.data_ptr(),
                                              sim._e_b_dev.data_ptr(), sim._uxb.data_ptr(), dom.epotRHS.data_ptr(), S),
            "current_lorentz": lambda: _lib.call("phb_current_lorentz", ct.byref(desc), dom.epotResult.data_ptr(),
                                                 sim._uxb.data_ptr(), sim._e_b_dev.data_ptr(), sim._stuart_dev.data_ptr(),
                                                 None, dom._src.data_ptr(), 1, S),
        }
        abytes = assembly_bytes(dims)
        if args.sweep_shear:
            # the same calls with phiPICT's non-orthogonal mode (cross terms in the matrices,
            # the explicit corner terms of the current results on the right-hand sides); their
            # fractions use the orthogonal kernels' byte counts, so they read as the cost of the
            # cross terms relative to the orthogonal assembly
            mode = backend.NON_ORTHO_CENTER_MATRIX | backend.NON_ORTHO_DIRECT_MATRIX | backend.NON_ORTHO_DIAGONAL_RHS
            kern.update({
                "advection_matrix (non-orthogonal)": lambda: backend.SetupAdvectionMatrix(dom, ts, mode),
                "advection_rhs (non-orthogonal)": lambda: backend.SetupAdvectionVelocity(dom, ts, mode, False),
                "pressure_matrix (non-orthogonal)": lambda: backend.SetupPressureMatrix(dom, ts, mode, False),
                "divergence (non-orthogonal)": lambda: backend.SetupPressureRHSdiv(dom, ts, mode),
            })
            for k in list(kern):
                if k.endswith("(non-orthogonal)"):
                    abytes[k] = abytes[k.split(" ")[0]]

        def timed(fn):
            ms = []
            for _ in range(reps):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                fn()
                e1.record()
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            return statistics.median(ms)

        for name, fn in kern.items():
            ms = timed(fn)
            gbs = abytes[name] * cells / (ms * 1e-3) / 1e9
            rows.append({"grid": f"{n}^{dims}", "cells": cells, "kernel": name, "bytes_per_cell": abytes[name],
                         "ms": round(ms, 4), "gbs": round(gbs, 1), "frac": round(gbs / peak, 3)})
        # Krylov iterations: fixed count, float32 (the refinement's inner solves)
        its = args.sweep_iterations
        P32 = backend._lo(dom, "P")
        C32 = backend._lo(dom, "C")
        amg = sim._amg_for("P", P32)
        bP = dom.pressureRHSdiv.float()
        bC = dom.velocityRHS.float()
        solves = [("cg_iteration", CG, 1, P32, bP, None, algorithmic_cg_bytes(dims, 4, 4)),
                  ("bicgstab_iteration", BICGSTAB, dims, C32, bC, None, 2 * (2 * dims + 1) * 4 + 18 * dims * 4)]
        if amg is not None:
            solves.append(("pcg_iteration", CG, 1, P32, bP, amg,
                           algorithmic_pcg_bytes(dims, amg.sizes[:amg.tail_level + 1], amg.coarse_inv.numel())))
        modes = args.sweep_modes.split(",")
        for name, kind, nrhs, A, b, mg, bpc in solves:
            s = solver_for(dom, kind, torch.float32, nrhs, tag="sweep-" + name)
            x = torch.zeros_like(b)
            for mode in modes:
                ms = []
                used = []
                for _ in range(reps):
                    x.zero_()
                    flush.zero_()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    s.solve(A, b, x, 1e-30, its, use_graph=MODES[mode], amg=mg)
                    e1.record()
                    e1.synchronize()
                    ms.append(e0.elapsed_time(e1))
                    used.append(max(i.usedIterations for i in s.results()))
                it = statistics.median(used)
                per = statistics.median(ms) / max(it, 1)
                gbs = bpc * cells / (per * 1e-3) / 1e9
                rows.append({"grid": f"{n}^{dims}", "cells": cells, "kernel": name + ("" if mode == "persistent" else f" ({mode})"),
                             "bytes_per_cell": round(bpc, 2), "ms": round(per, 4), "iterations": it, "gbs": round(gbs, 1),
                             "frac": round(gbs / peak, 3)})
        for r in rows[-(len(kern) + len(solves) * len(modes)):]:
            print(f"{r['grid']:>7} {r['kernel']:>20} {r['ms']:9.4f} ms {r['gbs']:8.1f} GB/s {r['frac']:6.3f}", file=sys.stderr)
        del sim, dom, kern
        torch.cuda.empty_cache()
    clk = clocks.stop()
    big = [r for r in rows if r["cells"] >= 16_000_000]
    return dict(metric="HBM roofline fraction (kernels of the step, grids >> L2)", value=round(min(r["frac"] for r in big), 3) if big else None,
                unit="fraction of measured HBM GB/s", n_gpus=world, steps=reps, warmup=args.warmup, higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype="f64 fields, f32 Krylov", data="synthetic (seeded)",
                config={"workload": "roofline sweep: " + ", ".join(f"{n}^{d}" for d, n in grids)
                        + (f" sheared x += {args.sweep_shear} y" if args.sweep_shear else "") + "; L2 flushed before every launch",
                        "parallelism": f"replicas x{world}"},
                clocks=clk, peak={"hbm_gbs": peak, "source": pk.get("source")}, sweep=rows, gpu_launches=None)


def run_adjoint(args, rank, world, local):
    """Gradient of L = ||u_outlet - target||^2 after the rollout with respect to the inflow
    profile (applied to inflow and outflow, which keeps the mass balance) and the Stuart
    number, by the hand-written adjoint; checked against fourth-order central differences
    on seeded directions (8 by default). Target: u_x = 1 - y^2 z^2 plus 1e-2 seeded noise on the outlet."""
    import phipict_b200 as pb
    from phipict_b200.adjoint import AdjointMHD, rollout

    wl = dict(WORKLOADS["adjoint"])
    if args.rollout:
        wl["rollout"] = args.rollout
    device = torch.device("cuda", local)
    dom = make_duct(device, torch.float64, wl["nx"], wl["ny"], wl["nz"], wl["nblocks"])
    dom.PrepareSolve()
    blocks = dom.getBlocks()
    N0 = wl["Ha"] ** 2 / wl["Re"]
    model = AdjointMHD(dom, wl["dt"], torch.tensor([N0]), torch.tensor([0.0, 1.0, 0.0], dtype=torch.float64),
                       steps=wl["rollout"], faces=[(blocks[0], "-x"), (blocks[-1], "+x")], checkpoint_every=wl["every"],
                       tol=wl["rtol"], mixed_precision=not args.plain_fp64)
    initial = model._state()
    last = blocks[-1]
    nx, ny, nz = last.getSizes()[:3]
    g = torch.Generator().manual_seed(7)
    yy = torch.linspace(-1, 1, ny, dtype=torch.float64).view(1, ny, 1)
    zz = torch.linspace(-1, 1, nz, dtype=torch.float64).view(nz, 1, 1)
    target = (1 - yy ** 2 * zz ** 2) + 1e-2 * torch.randn(nz, ny, 1, generator=g, dtype=torch.float64)
    target = target.to(device)
    n = dom.getTotalSize()

    def outlet(u):
        ux = u.view(3, n)[0][last.globalOffset:last.globalOffset + last.ncells()].view(nz, ny, nx)
        return ux[:, :, nx - 1:nx]

    def loss_of(u):
        return ((outlet(u) - target) ** 2).sum()

    p0 = model.faces[0]._velocity.detach().clone()
    prof = p0.clone().requires_grad_(True)
    N = torch.tensor([N0], dtype=torch.float64, requires_grad=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    u = rollout(model, prof, N, initial=[t.clone() for t in initial])
    L = loss_of(u)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    L.backward()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    checks = []
    for k in range(args.fd_directions):
        vp = torch.randn(p0.shape, generator=g, dtype=torch.float64).to(device)
        vp[:, 0] -= vp[:, 0].mean()
        vp[:, 1:] = 0
        vp /= vp.abs().max()  # unit max-norm direction: eps is the largest change of a face value
        vN = N0 * float(torch.randn(1, generator=g))  # the same relative size as the profile change
        eps = args.fd_eps

        def L_at(h):
            return float(loss_of(model.forward(p0 + h * vp, torch.tensor([N0 + h * vN]), [t.clone() for t in initial])))

        # fourth-order central difference: (8 (L(h) - L(-h)) - (L(2h) - L(-2h))) / 12h
        fd = (8 * (L_at(eps) - L_at(-eps)) - (L_at(2 * eps) - L_at(-2 * eps))) / (12 * eps)
        an = float((prof.grad * vp).sum()) + float(N.grad.reshape(-1)[0]) * vN
        checks.append({"analytic": an, "fd": fd, "rel_err": abs(an - fd) / max(abs(fd), 1e-300)})
    cells = dom.numCells()
    fwd, bwd = t1 - t0, t2 - t1
    return dict(metric="Mcell-steps/s", value=round(cells * wl["rollout"] / (fwd + bwd) / 1e6, 4), unit="Mcell-steps/s",
                n_gpus=world, steps=wl["rollout"], warmup=0, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f64 (adjoint kernels); solves " + ("f32 Krylov + f64 refinement" if not args.plain_fp64 else "f64"),
                data="synthetic (seeded inflow noise, seeded target)",
                config={"workload": f"adjoint: 2 blocks {wl['nx']}x{wl['ny']}x{wl['nz']} ({cells} cells), Ha {wl['Ha']}, "
                                    f"Re {wl['Re']}, {wl['rollout']} steps, checkpoints every {wl['every']}, rtol {wl['rtol']}",
                        "parallelism": f"replicas x{world}"},
                adjoint={"forward_s": round(fwd, 3), "backward_s": round(bwd, 3), "loss": float(L.detach()),
                         "grad_N": float(N.grad.reshape(-1)[0]), "grad_profile_norm": float(prof.grad.norm()),
                         "fd_checks": checks, "max_rel_err": max(c["rel_err"] for c in checks)},
                gpu_launches=None)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="duct3d", choices=list(WORKLOADS))
    ap.add_argument("--plain-fp64", action="store_true", help="the plain float64 path (no refinement)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-amg", action="store_true", help="unpreconditioned CG for pressure and potential")
    ap.add_argument("--no-fp64-leg", action="store_true", help="skip the plain FP64 comparison run")
    ap.add_argument("--pressure-warm-start", action="store_true",
                    help="start every pressure solve from the last step's pressure of the same corrector")
    ap.add_argument("--inner-rtol", type=float, default=None, help="inner FP32 reduction per refinement sweep")
    ap.add_argument("--no-alone", action="store_true", help="batch64: skip the one-at-a-time comparison")
    ap.add_argument("--no-batch64", action="store_true", help="duct3d: skip the batched-instances sub-record")
    ap.add_argument("--extrapolate-order", type=extrapolate_order, default="projection:12",
                    help="duct3d: degree m of the polynomial extrapolation of the pressure and potential "
                         "guesses from the last m+1 results, 'adaptive', or 'projection[:L]' (Galerkin "
                         "projection onto the last L results)")
    ap.add_argument("--no-extrapolate", dest="extrapolate", action="store_false",
                    help="duct3d: zero pressure guesses and the previous potential (phiPICT's defaults) instead of "
                         "guesses extrapolated from the last steps")
    ap.add_argument("--autotune", action="store_true",
                    help="tune the persistent Krylov kernels' CTAs per SM per solve during the warm-up")
    ap.add_argument("--requests", type=int, default=None, help="serve: number of requests")
    ap.add_argument("--plain-sample", type=int, default=8, help="serve: requests timed one at a time on plain FP64")
    ap.add_argument("--plain-steps", type=int, default=10, help="serve: timed steps per one-at-a-time request")
    ap.add_argument("--rollout", type=int, default=None, help="adjoint: steps of the differentiable rollout")
    ap.add_argument("--fd-directions", type=int, default=8, help="adjoint: random directions of the FD check")
    ap.add_argument("--fd-eps", type=float, default=3e-3, help="adjoint: central-difference step")
    ap.add_argument("--sweep-grids", default=None, help="sweep: grids as dims x n, e.g. 3x128,2x2048")
    ap.add_argument("--sweep-shear", type=float, default=0.0,
                    help="sweep: shear the grids (x += shear y) and also time the non-orthogonal assembly")
    ap.add_argument("--sweep-iterations", type=int, default=30, help="sweep: Krylov iterations per timed solve")
    ap.add_argument("--sweep-modes", default="persistent", help="sweep: solver launch modes (persistent, graph, host)")
    args = ap.parse_args()
    rank, world, local = dist_setup(args)
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    if args.workload == "batch64":
        line = run_batch64(args, rank, world, local)
    elif args.workload == "serve":
        line = run_serve(args, rank, world, local)
    elif args.workload == "adjoint":
        line = run_adjoint(args, rank, world, local)
    elif args.workload == "sweep":
        line = run_sweep(args, rank, world, local)
    else:
        line = run_ours(args, rank, world, local)
    if args.workload == "duct3d" and not args.no_batch64 and not args.plain_fp64:
        line["batch64"] = batch64_record(args, rank, world, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "duct3d":
        line["cpu_baseline"] = cpu_baseline(WORKLOADS[args.workload], 1, min_seconds=10.0)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
