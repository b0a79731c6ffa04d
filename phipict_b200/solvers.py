"""Batched Krylov solves of a domain's stencil matrices (the SolveLinear path of
solvers/linear_solve.cu:22-162 and the fused solvers of solvers/krylov/krylov.cu).

A :class:`StencilSolver` owns the device workspace of one solve configuration (solver
kind, dtype, right-hand sides per instance), so that its CUDA graph is built once and
relaunched with stable pointers; a :class:`RefinedSolver` runs FP32 inner solves inside
FP64 iterative refinement. Launches are asynchronous; :meth:`results` is the only call
that synchronises.
"""
from __future__ import annotations

import ctypes as ct
import enum
import os
from dataclasses import dataclass

import torch

from . import _lib
from .tolerance import to_device_tolerance

CG, BICGSTAB = 0, 1
STATUS = {0: "running", 1: "converged", 2: "non-finite", 3: "max iterations", 4: "rising"}

# Global solver settings (phiPICT's SetKrylovSettings, bindings.cpp:739-751): with graphs
# every solve is one CUDA-graph launch; without, every kernel is launched on its own and the
# host polls for completion every `check_interval` iterations (what a profiler needs).
# Solver launch modes: "persistent" (default) runs each Krylov solve as one cooperative
# kernel with grid barriers; "graph" as a conditional-WHILE CUDA graph of per-phase kernels;
# "host" launches every kernel on its own and polls; "persistent-host" keeps the persistent
# solves but runs the refinement's outer loop on the host. Kernel profilers cannot see
# kernels inside graphs with conditional nodes, so they need "host" or "persistent-host".
MODES = {"host": 0, "graph": 1, "persistent": 2, "persistent-host": 3}
SETTINGS = {
    "use_graphs": os.environ.get("PHIPICT_B200_GRAPHS", "1") != "0",
    "mode": os.environ.get("PHIPICT_B200_SOLVER_MODE", "persistent"),
    "check_interval": 8,
}
if not SETTINGS["use_graphs"]:
    SETTINGS["mode"] = "host"


def mode_code(use_graph=None) -> int:
    """phb_solve::use_graph for an explicit request (bool or mode code) or the settings."""
    if use_graph is None:
        return MODES[SETTINGS["mode"]]
    if isinstance(use_graph, bool):
        return 1 if use_graph else 0
    return int(use_graph)


@dataclass
class LinearSolverResultInfo:
    """Per right-hand-side outcome (bindings.cpp:727-732)."""
    finalResidual: float
    usedIterations: int
    converged: bool
    isFiniteResidual: bool
    status: int = 1
    innerIterations: int = 0

    def __str__(self) -> str:
        return (f"LinearSolverResultInfo(residual={self.finalResidual:.3e}, iterations={self.usedIterations}, "
                f"converged={self.converged}, finite={self.isFiniteResidual})")


class ConvergenceCriterion(enum.IntEnum):
    """Stop criteria of SolveLinear (solvers/linear_solvers.h:27-33). The Krylov solvers here
    test NORM2_NORMALIZED, ||r||_2 / sqrt(n) < tol; SolveLinear maps NORM2 onto it by scaling
    the tolerance, as phiPICT's fused solvers do (linear_solve.cu:48-55)."""
    NORM2 = 0
    NORM2_NORMALIZED = 1
    ABS_SUM = 2
    ABS_MEAN = 3
    ABS_MAX = 4


class LinsolveError(RuntimeError):
    """A linear solve did not converge (core/piso_diff.py:655-790)."""

    def __init__(self, message: str, infos: list[LinearSolverResultInfo] | None = None, tag: str = ""):
        super().__init__(message)
        self.infos = infos or []
        self.tag = tag


def _bytes(n: int, device: torch.device) -> torch.Tensor:
    return torch.zeros(max(256, int(n)), dtype=torch.uint8, device=device)


class StencilSolver:
    """CG or BiCGStab over all instances of a domain, ``nrhs`` right-hand sides each."""

    def __init__(self, domain, kind: int, dtype: torch.dtype, nrhs: int):
        self.domain = domain
        self.kind = kind
        self.dtype = dtype
        self.nrhs = nrhs
        lib = _lib.load()
        desc = domain.desc()
        dc = _lib.dtype_code(dtype)
        self.work = _bytes(lib.phb_solve_work_bytes(ct.byref(desc), kind, dc, nrhs), domain.getDevice())
        self.state = _bytes(lib.phb_solve_state_bytes(ct.byref(desc), nrhs), domain.getDevice())
        self._s = _lib.PhbSolve()
        self._keep = None

    def solve(self, A: torch.Tensor, b: torch.Tensor, x: torch.Tensor, tol, maxit: int,
              return_best: bool = False, use_graph: bool | None = None, amg=None, ctas_per_sm: int = 0) -> None:
        """Launch the solve of ``A x = b`` (x: initial guess, overwritten). Asynchronous.
        ``amg``: an :class:`~phipict_b200.amg.AmgHierarchy` set up for ``A`` (float32 CG
        with one right-hand side) preconditions every iteration with one V-cycle."""
        d = self.domain
        if A.dtype != self.dtype or b.dtype != self.dtype or x.dtype != self.dtype:
            raise TypeError("matrix, right-hand side and solution must share the solver dtype")
        if not (A.is_contiguous() and b.is_contiguous() and x.is_contiguous()):
            raise RuntimeError("solver operands must be contiguous")
        s = self._s
        s.kind = self.kind
        s.vec_dtype = s.mat_dtype = _lib.dtype_code(self.dtype)
        s.nrhs = self.nrhs
        s.maxit = int(maxit)
        s.return_best = int(bool(return_best)) if self.kind == CG else 0
        s.use_graph = mode_code(use_graph)
        s.check_every = int(SETTINGS["check_interval"])
        nsys = d.getBatchSize() * self.nrhs
        s.tol, self._keep = to_device_tolerance(tol, d.getDtype(), nsys, d.getDevice())
        s.A, s.b, s.x = A.data_ptr(), b.data_ptr(), x.data_ptr()
        s.work, s.state = self.work.data_ptr(), self.state.data_ptr()
        s.amg = amg.address() if amg is not None else None
        s.ctas_per_sm = int(ctas_per_sm)
        self._amg = amg
        _lib.call("phb_solve_run", ct.byref(d.desc()), ct.byref(s), _lib.stream_ptr(d.getDevice()))

    def results(self) -> list[LinearSolverResultInfo]:
        d = self.domain
        nsys = d.getBatchSize() * self.nrhs
        out = (_lib.PhbSolveResult * nsys)()
        _lib.call("phb_solve_results", ct.byref(d.desc()), ct.byref(self._s), out, _lib.stream_ptr(d.getDevice()))
        return [LinearSolverResultInfo(o.final_residual, o.used_iterations, bool(o.converged), bool(o.finite), o.status,
                                       o.inner_iterations) for o in out]


class RefinedSolver:
    """FP64 outer iterative refinement with FP32 inner CG/BiCGStab solves; the outer
    residual, the tolerance and the solution stay in FP64 on the device."""

    def __init__(self, domain, kind: int, nrhs: int, max_outer: int = 12, inner_rtol: float = 1e-4):
        if domain.getDtype() != torch.float64:
            raise TypeError("iterative refinement wraps float64 systems")
        self.domain = domain
        self.kind = kind
        self.nrhs = nrhs
        self.max_outer = max_outer
        self.inner_rtol = inner_rtol
        lib = _lib.load()
        desc = domain.desc()
        self.work = _bytes(lib.phb_refine_work_bytes(ct.byref(desc), kind, nrhs), domain.getDevice())
        self.state = _bytes(lib.phb_solve_state_bytes(ct.byref(desc), nrhs), domain.getDevice())
        self._r = _lib.PhbRefine()
        self._keep = None
        self.outer_used = 0

    def solve(self, A64: torch.Tensor, A32: torch.Tensor, b: torch.Tensor, x: torch.Tensor, tol, maxit: int,
              fetch: bool = False, amg=None, ctas_per_sm: int = 0) -> list[LinearSolverResultInfo] | None:
        """Launch the refined solve; ``amg`` (a hierarchy set up for ``A32``) preconditions
        the inner CG."""
        d = self.domain
        r = self._r
        r.kind = self.kind
        r.nrhs = self.nrhs
        r.max_outer = self.max_outer
        r.inner_maxit = int(maxit)
        r.inner_rtol = self.inner_rtol
        r.use_graph = mode_code()
        nsys = d.getBatchSize() * self.nrhs
        r.tol, self._keep = to_device_tolerance(tol, torch.float64, nsys, d.getDevice())
        r.A64, r.A32, r.b, r.x = A64.data_ptr(), A32.data_ptr(), b.data_ptr(), x.data_ptr()
        r.work, r.state = self.work.data_ptr(), self.state.data_ptr()
        r.amg = amg.address() if amg is not None else None
        r.ctas_per_sm = int(ctas_per_sm)
        self._amg = amg
        if not fetch:
            _lib.call("phb_refine_run", ct.byref(d.desc()), ct.byref(r), None, None, _lib.stream_ptr(d.getDevice()))
            return None
        out = (_lib.PhbSolveResult * nsys)()
        used = ct.c_int(0)
        _lib.call("phb_refine_run", ct.byref(d.desc()), ct.byref(r), out, ct.byref(used), _lib.stream_ptr(d.getDevice()))
        self.outer_used = used.value
        return [LinearSolverResultInfo(o.final_residual, o.used_iterations, bool(o.converged), bool(o.finite), o.status,
                                       o.inner_iterations) for o in out]

    def results(self) -> list[LinearSolverResultInfo]:
        """Outer results of the last solve (synchronises)."""
        d = self.domain
        nsys = d.getBatchSize() * self.nrhs
        out = (_lib.PhbSolveResult * nsys)()
        used = ct.c_int(0)
        _lib.call("phb_refine_results", ct.byref(d.desc()), ct.byref(self._r), out, ct.byref(used),
                  _lib.stream_ptr(d.getDevice()))
        self.outer_used = used.value
        return [LinearSolverResultInfo(o.final_residual, o.used_iterations, bool(o.converged), bool(o.finite), o.status,
                                       o.inner_iterations) for o in out]


class SolverTuner:
    """Per-solve tuning of the persistent Krylov kernels' grid (resident CTAs per SM), by
    measurement: the first ``trials`` x len(CANDIDATES) solves of each tag (``velocity``,
    ``pressure0``, ``epot``, ...) cycle through the candidates, each timed with CUDA events and
    divided by its iterations (the slowest system's; inner iterations under refinement); from
    then on the tag runs with the candidate of the lowest median time per iteration. 0 is the
    occupancy maximum (one CTA per tile where the grid allows), smaller values launch fewer,
    fuller CTAs. A choice changes the launch only, never the arithmetic: the results of every
    candidate are the same bits."""

    CANDIDATES = (0, 2, 1)

    def __init__(self, trials: int = 3):
        self.trials = int(trials)
        self.samples: dict[str, dict[int, list[float]]] = {}
        self.choice: dict[str, int] = {}

    def pick(self, tag: str) -> int:
        if tag in self.choice:
            return self.choice[tag]
        n = sum(len(v) for v in self.samples.get(tag, {}).values())
        return self.CANDIDATES[n % len(self.CANDIDATES)]

    def record(self, tag: str, candidate: int, ms: float, iterations: int) -> None:
        if tag in self.choice or iterations <= 0:
            return
        per = self.samples.setdefault(tag, {})
        per.setdefault(candidate, []).append(ms / iterations)
        if all(len(per.get(c, [])) >= self.trials for c in self.CANDIDATES):
            med = {c: sorted(v)[len(v) // 2] for c, v in per.items()}
            self.choice[tag] = min(med, key=med.get)

    def report(self) -> dict:
        out = {}
        for tag, per in self.samples.items():
            out[tag] = {"ctas_per_sm": self.choice.get(tag),
                        "us_per_iteration": {str(c): round(1e3 * sorted(v)[len(v) // 2], 3) for c, v in per.items()}}
        return out


def solver_for(domain, kind: int, dtype: torch.dtype, nrhs: int, tag: str = "") -> StencilSolver:
    key = ("krylov", kind, dtype, nrhs, tag)
    cache = domain.__dict__.setdefault("_solvers", {})
    s = cache.get(key)
    if s is None or s.domain is not domain:
        s = StencilSolver(domain, kind, dtype, nrhs)
        cache[key] = s
    return s


def refiner_for(domain, kind: int, nrhs: int, tag: str = "", **kw) -> RefinedSolver:
    key = ("refine", kind, nrhs, tag)
    cache = domain.__dict__.setdefault("_solvers", {})
    s = cache.get(key)
    if s is None:
        s = RefinedSolver(domain, kind, nrhs, **kw)
        cache[key] = s
    return s
