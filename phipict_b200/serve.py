"""Continuous batching of simulation requests: MHD cases of different grids and Hartmann
numbers advanced together in shared launches.

A :class:`Server` keeps the admitted requests of each dimensionality in one
:class:`~phipict_b200.batch.DomainBatch` (every kernel and every solve one launch for all of
them, fields and multigrid hierarchies resident on the device) and advances the batches one
PISO step per tick. Requests are admitted when they have arrived and their estimated
device memory fits the budget; finished requests leave after the step that completes them.
When the membership of a batch changes, the running instances' state (fields, solver warm
starts, velocity sources, the potential step's u x e_b) is copied out and into the new batch
exactly, so a request's result does not depend on the company it ran in: on the plain FP64
path it is bitwise the result it gets alone.

This is the serving loop of the reference's batching use (docs/source/batching.rst), which
can only batch copies of one domain; the request mix here may differ in grid, viscosity,
Stuart number, magnetic field and time step.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Callable

import torch

from .batch import DomainBatch
from .domain import Domain
from .mhd import MHDSimulation


@dataclass
class Request:
    """One simulation request: `build()` returns a prepared single-environment Domain."""
    rid: int
    build: Callable[[], Domain]
    stuart: float
    e_b: tuple[float, float, float]
    steps: int
    dt: float
    arrival: float = 0.0           # seconds after the server starts
    cost_hint: float | None = None  # estimated work (cells x steps) for routing; None: 1
    # filled by the server
    domain: Domain | None = None
    uxb: torch.Tensor | None = None
    done: int = 0
    admitted: float | None = None
    finished: float | None = None
    cells: int = 0
    failed: str | None = None

    @property
    def latency(self) -> float | None:
        return None if self.finished is None else self.finished - self.arrival


def estimate_bytes(domain: Domain) -> int:
    """Device bytes a request holds while it runs (fields, stencils, solver and multigrid
    work): about 60 values of its dtype per cell and spatial dimension, plus the float32
    copies; a conservative admission estimate, not an allocator query."""
    item = torch.finfo(domain.getDtype()).bits // 8
    return int(domain.numCells() * domain.getSpatialDims() * (60 * item + 40))


@dataclass
class _Group:
    dims: int
    requests: list[Request] = field(default_factory=list)
    batch: DomainBatch | None = None
    sim: MHDSimulation | None = None
    batch_requests: list[Request] = field(default_factory=list)  # instance order of `batch`
    dirty: bool = True


class Server:
    """Continuous-batching MHD request loop on one device.

    sim_kwargs: keyword arguments of every batch's MHDSimulation (tolerances, precision,
    multigrid). hbm_budget: bytes of device memory the running requests may hold."""

    def __init__(self, device="cuda", hbm_budget: float = 150e9, max_instances: int = 64, sim_kwargs: dict | None = None,
                 clock: Callable[[], float] | None = None):
        self.device = torch.device(device)
        self.hbm_budget = float(hbm_budget)
        self.max_instances = int(max_instances)
        self.sim_kwargs = dict(sim_kwargs or {})
        self.clock = clock or time.perf_counter
        self.pending: list[Request] = []
        self.groups: dict[int, _Group] = {}
        self.finished: list[Request] = []
        self.held = 0
        self.peak_held = 0
        self.steps_run = 0
        self.cell_steps = 0
        self.joins = 0    # admissions into a batch that was already running
        self.repacks = 0  # batch rebuilds after a membership change
        self._t0 = None

    # --- admission ------------------------------------------------------------------------
    def submit(self, req: Request) -> None:
        self.pending.append(req)
        self.pending.sort(key=lambda r: r.arrival)

    def _now(self) -> float:
        return self.clock() - self._t0

    def _admit(self, now: float) -> None:
        running = sum(len(g.requests) for g in self.groups.values())
        keep = []
        for req in self.pending:
            if req.arrival > now or running >= self.max_instances:
                keep.append(req)
                continue
            if req.domain is None:
                req.domain = req.build()
                if not req.domain.IsInitialized():
                    req.domain.PrepareSolve()
            need = estimate_bytes(req.domain)
            if need > self.hbm_budget:  # can never run: refuse instead of waiting forever
                req.failed = "the request exceeds the memory budget"
                req.finished = now
                self.finished.append(req)
                continue
            if self.held + need > self.hbm_budget:
                keep.append(req)
                continue
            self.held += need
            self.peak_held = max(self.peak_held, self.held)
            req.cells = req.domain.numCells()
            req.admitted = now
            g = self.groups.setdefault(req.domain.getSpatialDims(), _Group(req.domain.getSpatialDims()))
            if g.requests:  # joins a batch that is already running
                self.joins += 1
            g.requests.append(req)
            g.dirty = True
            running += 1
        self.pending = keep

    # --- batches --------------------------------------------------------------------------
    def _stash(self, g: _Group) -> None:
        """Copy the running batch's state back to its requests."""
        if g.batch is None:
            return
        g.batch.scatter()
        for k, req in enumerate(g.batch_requests):
            req.uxb = g.sim._uxb[g.batch.instance_slice(k, 3)].clone()

    def _repack(self, g: _Group) -> None:
        self._stash(g)
        g.batch = g.sim = None
        if not g.requests:
            g.dirty = False
            return
        self.repacks += 1
        reqs = list(g.requests)
        batch = DomainBatch([r.domain for r in reqs])
        dt = torch.tensor([r.dt for r in reqs], dtype=torch.float64)
        stuart = torch.tensor([r.stuart for r in reqs], dtype=torch.float64)
        e_b = torch.tensor([r.e_b for r in reqs], dtype=torch.float64)
        sim = MHDSimulation(batch, float(dt[0]), stuart, e_b, **self.sim_kwargs)
        sim.time_step = dt if len(set(float(v) for v in dt)) > 1 else float(dt[0])
        for k, req in enumerate(reqs):
            if req.uxb is not None:
                sim._uxb[batch.instance_slice(k, 3)].copy_(req.uxb)
        g.batch, g.sim, g.batch_requests = batch, sim, reqs
        g.dirty = False

    @staticmethod
    def _failed_instances(g: _Group) -> set[int]:
        """Instances of the batch with a solve that did not converge in the last step (the
        others' results are unaffected: every system of a batch is solved on its own)."""
        B = g.batch.getBatchSize()
        bad = set()
        for tag, infos in g.sim.solve_report():
            per = max(1, len(infos) // B)
            for i, inf in enumerate(infos):
                if not inf.converged and not (tag.startswith("epot") and g.sim._accept_best(inf)):
                    bad.add(i // per)
        return bad if bad else set(range(B))

    def _retire(self, g: _Group, now: float) -> None:
        done = [r for r in g.requests if r.done >= r.steps or r.failed]
        if not done:
            return
        self._stash(g)
        for r in done:
            r.finished = now
            g.requests.remove(r)
            self.held -= estimate_bytes(r.domain)
            self.finished.append(r)
        g.dirty = True
        g.batch = g.sim = None

    # --- the loop ---------------------------------------------------------------------------
    def tick(self) -> bool:
        """Admit, advance every batch one step, retire. False when there is nothing to do."""
        if self._t0 is None:
            self._t0 = self.clock()
        now = self._now()
        self._admit(now)
        active = [g for g in self.groups.values() if g.requests]
        if not active:
            if not self.pending:
                return False
            wait = self.pending[0].arrival - now
            if wait > 0:
                time.sleep(min(wait, 0.05))
            return True
        for g in active:
            if g.dirty or g.sim is None:
                self._repack(g)
            ok = g.sim.single_step()
            self.steps_run += 1
            bad = set() if ok else self._failed_instances(g)
            for k, r in enumerate(g.batch_requests):
                r.done += 1
                self.cell_steps += r.cells
                if k in bad:
                    r.failed = g.sim.last_error or "step failed"
        now = self._now()
        for g in active:
            self._retire(g, now)
        return True

    def run(self, requests: list[Request] | None = None) -> dict:
        for r in requests or []:
            self.submit(r)
        self._t0 = self.clock()
        while self.tick():
            pass
        return self.report()

    def report(self) -> dict:
        lat = sorted(r.latency for r in self.finished if r.latency is not None)
        wall = self._now() if self._t0 is not None else 0.0
        return {"requests": len(self.finished), "failed": sum(1 for r in self.finished if r.failed),
                "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99), "wall_s": wall,
                "mcell_steps_per_s": self.cell_steps / wall / 1e6 if wall > 0 else None,
                "batch_steps": self.steps_run, "peak_held_bytes": self.peak_held,
                "joins": self.joins, "repacks": self.repacks,
                "latencies": lat, "cell_steps": self.cell_steps, "cells_total": sum(r.cells for r in self.finished)}


def percentile(sorted_values: list[float], p: float) -> float | None:
    """The nearest-rank p-th percentile of an ascending list (None when empty)."""
    if not sorted_values:
        return None
    k = min(len(sorted_values) - 1, max(0, math.ceil(p / 100 * len(sorted_values)) - 1))
    return sorted_values[k]


def route(requests: list[Request], world: int) -> list[list[Request]]:
    """Assign a request stream to `world` servers, one per GPU: in arrival order, each request
    goes to the server with the least estimated work so far (cost_hint, or 1 per request;
    ties to the lower rank). Deterministic, so every rank computes the same assignment from
    the same stream without exchanging anything."""
    load = [0.0] * world
    out: list[list[Request]] = [[] for _ in range(world)]
    for req in sorted(requests, key=lambda r: (r.arrival, r.rid)):
        k = min(range(world), key=lambda i: (load[i], i))
        out[k].append(req)
        load[k] += req.cost_hint if req.cost_hint is not None else 1.0
    return out


def merge_reports(reports: list[dict]) -> dict:
    """One report for the whole job from the servers' reports: latency percentiles over all
    requests, cell-steps of all servers over the longest wall time."""
    lat = sorted(x for r in reports for x in r["latencies"])
    wall = max(r["wall_s"] for r in reports)
    cell_steps = sum(r["cell_steps"] for r in reports)
    return {"requests": sum(r["requests"] for r in reports), "failed": sum(r["failed"] for r in reports),
            "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99), "wall_s": wall,
            "mcell_steps_per_s": cell_steps / wall / 1e6 if wall > 0 else None,
            "batch_steps": sum(r["batch_steps"] for r in reports),
            "joins": sum(r.get("joins", 0) for r in reports), "repacks": sum(r.get("repacks", 0) for r in reports),
            "peak_held_bytes": max(r["peak_held_bytes"] for r in reports),
            "latencies": lat, "cell_steps": cell_steps, "cells_total": sum(r["cells_total"] for r in reports),
            "servers": len(reports)}


def gather_reports(report: dict, world: int) -> dict:
    """The merged report of all ranks' servers (every rank gets it); the report itself when
    there is one rank. Uses the default process group."""
    if world == 1:
        return merge_reports([report])
    import torch.distributed as dist

    reports: list = [None] * world
    dist.all_gather_object(reports, report)
    return merge_reports(reports)


def poisson_arrivals(n: int, rate: float, seed: int) -> list[float]:
    """Arrival times (s) of a seeded Poisson process of the given rate."""
    g = torch.Generator().manual_seed(seed)
    gaps = -torch.log(torch.rand(n, generator=g, dtype=torch.float64)) / rate
    return torch.cumsum(gaps, 0).tolist()


__all__ = ["Request", "Server", "estimate_bytes", "gather_reports", "merge_reports", "percentile", "poisson_arrivals", "route"]
