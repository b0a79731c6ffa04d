"""PISO simulation driver (phiPICT core/piso_simulation.py and simulation/simulation.py).

``Simulation`` keeps phiPICT's constructor keywords and step semantics: one PISO step is
the momentum predictor (advection matrix, right-hand side, BiCGStab solve warm-started
from the last velocity), ``corrector_steps`` pressure correctors (pressure system, CG
solve, mean projection, velocity correction) and the copy of the result to the blocks,
with the same hook points (core/piso_simulation.py:3525-4169).

What changes is the execution: every stage is a stream-ordered launch of the phipict_b200
kernels with no host synchronisation inside the step; each solve is one CUDA-graph launch
(or a node of a graph the caller is capturing). The solver outcomes are read back once at
the end of the step, where phiPICT reads them after every solve.

Extensions (keyword arguments phiPICT does not have):
  ``mixed_precision``: with a float64 domain, every solve runs FP32 Krylov iterations
      inside FP64 iterative refinement to the requested tolerance.
  ``check_solves``: read the solver outcomes at the end of every step (default True).
      With False the step never synchronises; failures surface through
      :meth:`solve_report`.
  ``autotune_solvers``: measure and pick the CTAs per SM of each solve (SolverTuner).
  ``extrapolate_guesses``: start the pressure and potential solves from a polynomial
      extrapolation of their last results (a degree m >= 1, True: 1, or "adaptive") or from
      the Galerkin projection onto the span of the last L results ("projection[:L]", 12).
"""
from __future__ import annotations

import math

from typing import Any, Literal

import numpy as np
import torch

from . import _C as backend
from .domain import Domain, FixedBoundary
from .hooks import Hook, Hooks
from .solvers import BICGSTAB, CG, LinearSolverResultInfo, LinsolveError, SolverTuner, refiner_for, solver_for
from .tolerance import SolverTolerance, coerce_tolerance

_UNSUPPORTED_TRUE = ("scipy_solve_advection", "scipy_solve_pressure", "differentiable_unsupported")


def extrapolate_into(x: torch.Tensor, hist: list, order: int) -> None:
    """x holds the last result x_n; hist the ones before it (x_(n-1), x_(n-2), ..., newest
    first). Overwrite x with the polynomial extrapolation of the highest order m <= `order`
    that the history allows: sum over k = 0..m of (-1)^k binom(m+1, k+1) x_(n-k) (m = 1:
    2 x_n - x_(n-1); m = 2: 3 x_n - 3 x_(n-1) + x_(n-2))."""
    hist = [h for h in hist if h.shape == x.shape]
    m = min(order, len(hist))
    if m < 1:
        return
    x.mul_(float(math.comb(m + 1, 1)))
    for k in range(1, m + 1):
        x.add_(hist[k - 1], alpha=float((-1) ** k * math.comb(m + 1, k + 1)))


def push_history(hist: list, x: torch.Tensor, order: int, spare: list | None = None) -> None:
    """Prepend a copy of x (the result before the newest), keeping `order` entries; new
    entries come from `spare` (buffers allocated up front) while it has any."""
    if len(hist) < order:
        if spare:
            buf = spare.pop()
            buf.copy_(x)
            hist.insert(0, buf)
        else:
            hist.insert(0, x.clone())
        return
    buf = hist.pop()
    buf.copy_(x)
    hist.insert(0, buf)


class GuessExtrapolator:
    """Initial guesses of one recurring solve (the pressure of one corrector, the potential)
    from its results of the last steps. Fixed order m: the polynomial extrapolation of degree
    m (extrapolate_into). Adaptive: after each solve, the extrapolations of every degree up to
    `max_order` are compared with the new result on the device, and the next solve uses the
    degree that predicted it best (the error norms come back through pinned memory after an
    event and are read at the next guess, so the choice adds no wait on the GPU)."""

    def __init__(self, max_order: int, adaptive: bool):
        self.max_order = int(max_order)
        self.adaptive = bool(adaptive)
        self.order = 1 if adaptive else self.max_order
        self.hist: list[torch.Tensor] = []
        self.last: torch.Tensor | None = None
        self._spare: list[torch.Tensor] = []  # history buffers not in use yet
        self._errs = None  # (host norms, event or None) of the last comparison

    def guess(self, x: torch.Tensor, A=None, b=None, domain=None) -> bool:
        """Write the guess into x (the system's A and b are not needed); False when there is
        no previous result yet."""
        if self.last is None or self.last.shape != x.shape:
            return False
        if self._errs is not None:
            host, ev = self._errs
            if ev is not None:
                ev.synchronize()
            self.order = int(torch.argmin(host).item())
            self._errs = None
        x.copy_(self.last)
        extrapolate_into(x, self.hist, self.order)
        return True

    def _compare(self, result: torch.Tensor) -> None:
        # guesses of every degree from the backward differences of (last, hist...):
        # degree m = sum over j <= m of the j-th backward difference at the last result
        vals = [self.last] + [h for h in self.hist if h.shape == result.shape][: self.max_order]
        g = torch.empty((len(vals),) + tuple(result.shape), dtype=result.dtype, device=result.device)
        g[0].copy_(self.last)
        row = vals
        for m in range(1, len(vals)):
            row = [row[i] - row[i + 1] for i in range(len(row) - 1)]
            torch.add(g[m - 1], row[0], out=g[m])
        errs = torch.linalg.vector_norm((g - result).reshape(len(vals), -1), dim=1)
        if result.is_cuda:
            host = torch.empty(errs.shape, dtype=errs.dtype, pin_memory=True)
            host.copy_(errs, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record()
            self._errs = (host, ev)
        else:
            self._errs = (errs, None)

    def update(self, result: torch.Tensor) -> None:
        """Record the result of the solve."""
        if self.last is not None and self.last.shape == result.shape:
            if self.adaptive:
                self._compare(result)
            push_history(self.hist, self.last, self.max_order, self._spare)
            self.last.copy_(result)
        else:
            # every buffer is allocated with the first result, none in later steps
            self.hist.clear()
            self.last = result.clone()
            self._spare = [torch.empty_like(result) for _ in range(self.max_order)]


class ProjectedGuess:
    """Initial guesses of one recurring solve as the Galerkin projection of its solution onto
    the span of its last `size` results (P. F. Fischer, "Projection techniques for iterative
    solution of Ax = b with successive right-hand sides", Comput. Methods Appl. Mech. Engrg.
    163, 1998): x0 = V alpha with (V^T A V) alpha = V^T b, for a symmetric definite A the
    A-norm-best guess in that span, so never worse in that norm than a polynomial
    extrapolation of the same results. The basis rows are the backward differences of the
    results (x_n, x_n - x_(n-1), ...: the same span, far better conditioned than the results
    themselves) in one float64 (size, cells) buffer; A V is taken with the current matrix
    (phb_stencil_apply), G = V (A V)^T and c = V b in one pass (phb_projection_gram) and the
    size x size system solved on the device (phb_projection_solve), so a guess adds no host
    synchronisation. `apply` and `solve` replace those calls: (A, V, Y, m) -> Y[:m] = A V[:m]
    and (G, c) -> alpha."""

    REG = 1e-13

    def __init__(self, size: int, apply=None, solve=None):
        if not 1 <= int(size) <= 16:
            raise ValueError("a projected guess takes 1 to 16 basis vectors")
        self.size = int(size)
        self.n = 0
        self.D: torch.Tensor | None = None
        self._Dn = self._Y = self._alpha = None
        self._apply, self._solve = apply, solve

    def guess(self, x: torch.Tensor, A=None, b=None, domain=None) -> bool:
        """Write the guess into x for the system A x = b; False before the first result."""
        if self.n == 0 or self.D.shape[1] != x.numel():
            return False
        m = self.n
        V, Y = self.D[:m], self._Y[:m]
        if self._apply is not None:
            self._apply(A, V, Y, m)
        else:
            import ctypes as ct

            from . import _lib

            if A.dtype != torch.float64:
                raise ValueError("projected guesses need a float64 matrix")
            if x.numel() != int(domain.desc().ncells) or b.numel() != x.numel():
                raise ValueError("projected guesses need one value per cell in x and b")
            _lib.call("phb_stencil_apply", ct.byref(domain.desc()), A.data_ptr(), V.data_ptr(), Y.data_ptr(), m,
                      V.stride(0), _lib.stream_ptr(x.device))
        if self._solve is not None:
            alpha = self._solve(torch.mm(V, Y.t()), torch.mv(V, b.reshape(-1)))
        else:
            from . import _lib

            if not b.is_contiguous():
                raise ValueError("projected guesses need a contiguous right-hand side")
            st = _lib.stream_ptr(x.device)
            G, c, alpha = self._gram[: m * m], self._gram[m * m: m * m + m], self._alpha[:m]
            _lib.call("phb_projection_gram", V.data_ptr(), Y.data_ptr(), b.data_ptr(), m, V.shape[1], V.stride(0),
                      G.data_ptr(), c.data_ptr(), st)
            _lib.call("phb_projection_solve", G.data_ptr(), c.data_ptr(), m, self.REG, alpha.data_ptr(), st)
        torch.mv(V.t(), alpha, out=x.view(-1))
        return True

    def update(self, result: torch.Tensor) -> None:
        """Record the result of the solve: the new rows are D'_0 = x and
        D'_j = x - (D_0 + ... + D_(j-1)), the oldest row dropped when the basis is full."""
        v = result.reshape(-1)
        if self.D is None or self.D.shape[1] != v.numel():
            # rows a multiple of four values apart (the stencil product's vector loads)
            n, stride = v.numel(), (v.numel() + 3) // 4 * 4
            self.D, self._Dn, self._Y = (torch.empty(self.size, stride, dtype=torch.float64, device=v.device)[:, :n]
                                         for _ in range(3))
            self._alpha = torch.empty(self.size, dtype=torch.float64, device=v.device)
            self._gram = torch.empty(self.size * self.size + self.size, dtype=torch.float64, device=v.device)
            self.n = 0
        k = min(self.n + 1, self.size)
        if k > 1:
            torch.cumsum(self.D[: k - 1], 0, out=self._Y[: k - 1])
            torch.sub(v.unsqueeze(0), self._Y[: k - 1], out=self._Dn[1:k])
        self._Dn[0].copy_(v)
        self.D, self._Dn = self._Dn, self.D
        self.n = k


class Simulation:
    """A drop-in for ``phipict.Simulation`` on phipict_b200 kernels."""

    # pressure systems at least this large use the multigrid preconditioner when
    # pressure_use_amg is None (core/piso_simulation.py:1118-1122)
    PRESSURE_AMG_AUTO_MIN_ROWS = 200_000
    PRESSURE_AMG_AUTO_MIN_ROWS_BATCHED = 400_000

    def __init__(
        self,
        domain: Domain,
        dt: float,
        substeps: int | Literal["ADAPTIVE"] = 1,
        corrector_steps: int = 2,
        density_viscosity: float | None = None,
        adaptive_CFL: float = 0.8,
        adaptive_CFL_per_env: bool = True,
        prep_fn: Hooks | dict | None = None,
        advection_use_BiCG: bool = True,
        pressure_use_BiCG: bool = False,
        scipy_solve_advection: bool = False,
        scipy_solve_pressure: bool = False,
        preconditionBiCG: bool = False,
        BiCG_precondition_fallback: bool = True,
        advection_tol: float | SolverTolerance | None = None,
        pressure_tol: float | SolverTolerance | None = None,
        pressure_tol_intermediate: float | SolverTolerance | None = None,
        pressure_warm_start: bool = False,
        pressure_use_amg: bool | None = None,
        pressure_amg_options: dict | None = None,
        flux_balance_tol: float = 1e-5,
        convergence_tol: float | None = None,
        solver_double_fallback: bool = False,
        advect_non_ortho_steps: int = 1,
        pressure_non_ortho_steps: int = 1,
        normalize_pressure_result: bool = True,
        pressure_return_best_result: bool = False,
        advect_passive_scalar: bool = True,
        pressure_time_step_normalized: bool = False,
        velocity_corrector: str = "FD",
        non_orthogonal: bool = True,
        differentiable: bool = False,
        exclude_advection_solve_gradients: bool = False,
        exclude_pressure_solve_gradients: bool = False,
        output_resampling_shape: tuple[int, ...] | None = None,
        output_resampling_fill_max_steps: int = 0,
        hooks: Hooks | dict | None = None,
        mixed_precision: bool = False,
        check_solves: bool = True,
        autotune_solvers: bool = False,
        extrapolate_guesses: bool | int | str = False,
    ) -> None:
        if hooks is not None and prep_fn is not None:
            raise ValueError("Pass hooks or its former name prep_fn, not both.")
        if scipy_solve_advection or scipy_solve_pressure:
            raise NotImplementedError("SciPy solves are not part of the phipict_b200 GPU path")
        if velocity_corrector != "FD":
            raise NotImplementedError("phipict_b200 implements the finite-difference velocity corrector ('FD')")
        if pressure_time_step_normalized:
            raise NotImplementedError("pressure_time_step_normalized is not implemented")
        if substeps != "ADAPTIVE" and not (isinstance(substeps, int) and substeps > 0):
            raise ValueError("substeps must be a positive int or 'ADAPTIVE'")
        self.domain = domain
        self.time_step = float(dt)
        self.substeps = substeps if substeps == "ADAPTIVE" else int(substeps)
        self.adaptive_CFL = float(adaptive_CFL)
        self.adaptive_CFL_per_env = bool(adaptive_CFL_per_env)
        self.corrector_steps = int(corrector_steps)
        self.density_viscosity = density_viscosity
        self.hooks = Hooks.coerce(hooks if hooks is not None else prep_fn)
        self.advection_use_BiCG = advection_use_BiCG
        self.pressure_use_BiCG = pressure_use_BiCG
        self.advection_tol = coerce_tolerance(advection_tol)
        self.pressure_tol = coerce_tolerance(pressure_tol)
        self.pressure_tol_intermediate = coerce_tolerance(pressure_tol_intermediate)
        self.pressure_warm_start = pressure_warm_start
        self.pressure_use_amg = pressure_use_amg
        self._pressure_amg_options = dict(pressure_amg_options or {})
        self._amg_cache: dict = {}
        self.flux_balance_tol = flux_balance_tol
        self.convergence_tol = convergence_tol
        self.normalize_pressure_result = normalize_pressure_result
        self.pressure_return_best_result = pressure_return_best_result
        self.non_orthogonal = non_orthogonal
        self.advect_passive_scalar = bool(advect_passive_scalar)
        # differentiable=True: every PISO step is one torch.autograd node whose backward is the
        # hand-written adjoint of the step (phipict_b200.differentiable); set up at the first step
        self.differentiable = bool(differentiable)
        self._diff = None
        self.linear_solve_max_iterations = 5000
        self.mixed_precision = bool(mixed_precision)
        # mixed precision: each inner FP32 solve reduces the outer residual by this factor
        self.refinement_inner_rtol = 1e-4
        # grid of the persistent Krylov kernels tuned per solve by measurement (SolverTuner)
        self.solver_tuner = SolverTuner() if autotune_solvers else None
        # initial guesses of the pressure (per corrector) and potential solves from the last
        # steps' results: a polynomial extrapolation of degree m >= 1 (True: 1) or "adaptive"
        # (the degree up to 4 that predicted the last result best), GuessExtrapolator; or
        # "projection[:L]", the Galerkin projection onto the last L (12) results, ProjectedGuess
        mode = extrapolate_guesses
        adaptive = mode == "adaptive"
        self._guess_projection = 0
        if isinstance(mode, str) and mode.startswith("projection"):
            self._guess_projection = int(mode.split(":", 1)[1]) if ":" in mode else 12
            ProjectedGuess(self._guess_projection)  # checks the size
            if domain.getDtype() != torch.float64:
                raise ValueError("extrapolate_guesses='projection' needs a float64 domain")
            mode = 1
        self.extrapolate_guesses = 4 if adaptive else int(mode)
        self._extrapolate_adaptive = adaptive
        self._pressure_extrap: dict[int, GuessExtrapolator | ProjectedGuess] = {}
        self.check_solves = check_solves
        self.total_step = 0
        self.total_time = 0.0
        self._pressure_guess: dict[int, torch.Tensor] = {}
        self._pending: list[tuple[str, Any]] = []
        self._tuning: list = []  # (index in _pending, tag, (candidate, start event, end event))
        self._last_report: list[tuple[str, list[LinearSolverResultInfo]]] = []
        self._flux_checked_version = -1
        self._solve_events: list | None = None  # (start, end) CUDA events per solve when a list
        self.last_error: str | None = None
        if not domain.IsInitialized():
            domain.PrepareSolve()
        if self.mixed_precision and domain.getDtype() != torch.float64:
            raise TypeError("mixed_precision refines float64 systems; create the domain with dtype=torch.float64")
        domain._mixed = self.mixed_precision
        if pressure_use_amg and not self._amg_dtype_ok():
            raise NotImplementedError("the multigrid V-cycle runs in float32: use a float32 domain or mixed_precision=True")
        if int(advect_non_ortho_steps) < 0 or int(pressure_non_ortho_steps) < 0:
            raise ValueError("advect_non_ortho_steps and pressure_non_ortho_steps must not be negative")
        self.advect_non_ortho_steps = int(advect_non_ortho_steps)
        self.pressure_non_ortho_steps = int(pressure_non_ortho_steps)

    # --- helpers ---------------------------------------------------------------------
    # core/piso_simulation.py:1124-1126: the flags of the non-orthogonal mode
    NON_ORTHO_MODE = backend.NON_ORTHO_CENTER_MATRIX | backend.NON_ORTHO_DIRECT_MATRIX | backend.NON_ORTHO_DIAGONAL_RHS

    def _nonortho_flags(self) -> int:
        """The non-orthogonal flags of this step: phiPICT's mode when ``non_orthogonal`` is set
        and the grid has cross terms (without them every non-orthogonal term is exactly zero
        and the orthogonal step gives the same result), else 0."""
        if not self.non_orthogonal or self.domain.getSpatialDims() < 2:
            return 0
        return self.NON_ORTHO_MODE if self.domain.hasNonOrthogonalMetrics() else 0

    def _time_step_tensor(self, time_step: float | torch.Tensor | None) -> torch.Tensor:
        if time_step is None:
            time_step = self.time_step
        if isinstance(time_step, torch.Tensor):
            return time_step.detach().reshape(-1).to("cpu", torch.float64)
        return torch.tensor([float(time_step)], dtype=torch.float64)

    def _run_hooks(self, hook: Hook, **kw) -> None:
        if self.hooks:
            self.hooks.run(hook, domain=self.domain, total_step=self.total_step, total_time=self.total_time, **kw)

    def _pressure_tol_for(self, cstep: int):
        if self.pressure_tol_intermediate is None or cstep == self.corrector_steps - 1:
            return self.pressure_tol
        return self.pressure_tol_intermediate

    def _new_guess(self) -> GuessExtrapolator | ProjectedGuess:
        """The initial-guess state of one recurring solve (extrapolate_guesses)."""
        if self._guess_projection:
            return ProjectedGuess(self._guess_projection)
        return GuessExtrapolator(self.extrapolate_guesses, self._extrapolate_adaptive)

    def solve(self, which: str, rhs: torch.Tensor, x: torch.Tensor, *, use_BiCG: bool, tol, tag: str,
              nrhs: int = 1, return_best: bool = False, max_iter: int | None = None) -> None:
        """Launch one solve of a domain matrix (stencil) into ``x`` (the initial guess)."""
        d = self.domain
        maxit = self.linear_solve_max_iterations if max_iter is None else int(max_iter)
        kind = BICGSTAB if use_BiCG else CG
        ev = None
        if self._solve_events is not None:
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True), tag)
            ev[0].record()
            self._solve_events.append(ev)
        self._solve_launch(which, rhs, x, kind, tol, tag, nrhs, return_best, maxit)
        if ev is not None:
            ev[1].record()

    def _solve_launch(self, which, rhs, x, kind, tol, tag, nrhs, return_best, maxit) -> None:
        d = self.domain
        pc = kind == CG and nrhs == 1 and self._amg_wanted(which)
        tune = None
        ctas = 0
        if self.solver_tuner is not None:
            ctas = self.solver_tuner.pick(tag)
            tune = (ctas, torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            tune[1].record()
        if self.mixed_precision:
            lo = backend._lo(d, which)
            amg = self._amg_for(which, lo) if pc else None
            r = refiner_for(d, kind, nrhs, tag=tag)
            r.inner_rtol = self.refinement_inner_rtol
            r.solve(d._stencil(which), lo, rhs, x, tol, maxit, amg=amg, ctas_per_sm=ctas)
            solver = r
        else:
            A = d._stencil(which)
            amg = self._amg_for(which, A) if pc else None
            solver = solver_for(d, kind, d.getDtype(), nrhs, tag=tag)
            solver.solve(A, rhs, x, tol, maxit, return_best=return_best, amg=amg, ctas_per_sm=ctas)
        if tune is not None:
            tune[2].record()
            self._tuning.append((len(self._pending), tag, tune))
        self._pending.append((tag, solver))

    # --- multigrid preconditioner ------------------------------------------------------
    def _amg_dtype_ok(self) -> bool:
        return self.domain.getDtype() == torch.float32 or self.mixed_precision

    def _amg_wanted(self, which: str) -> bool:
        """pressure_use_amg: True/False, or None for automatic from PRESSURE_AMG_AUTO_MIN_ROWS
        unknowns (core/piso_simulation.py:2222-2300)."""
        if which != "P" or self.pressure_use_BiCG or not self._amg_dtype_ok():
            return False
        use = self.pressure_use_amg
        if use is None:
            d = self.domain
            rows = d.numCells()
            limit = self.PRESSURE_AMG_AUTO_MIN_ROWS if d.getBatchSize() == 1 else self.PRESSURE_AMG_AUTO_MIN_ROWS_BATCHED
            return rows >= limit
        return bool(use)

    def _amg_options(self, which: str) -> dict:
        return self._pressure_amg_options

    def _amg_for(self, which: str, A32: torch.Tensor):
        """The multigrid hierarchy of matrix `which`, or None for a grid that cannot be
        coarsened (single cells, or a coarsest level above the dense limit): plain CG then."""
        from .amg import hierarchy_for

        d = self.domain
        if self._amg_cache.get(("unavailable", which)) is d._blocks_dev:
            return None
        try:
            # the pressure matrix changes every step: phiPICT's default coarse_refresh_interval
            # of 4 for it (core/piso_simulation.py:2268)
            return hierarchy_for(d, which, A32, d._matrix_version(which), self._amg_cache, self._amg_options(which),
                                 coarse_refresh_interval=4 if which == "P" else 1)
        except ValueError:
            self._amg_cache[("unavailable", which)] = d._blocks_dev
            return None

    def collect_solves(self, raise_on_failure: bool = True) -> bool:
        """Read the outcomes of the solves launched since the last call (synchronises)."""
        ok = True
        report = []
        for tag, s in self._pending:
            infos = s.results()
            report.append((tag, infos))
            good = all(i.converged or (tag.startswith("epot") and self._accept_best(i)) for i in infos)
            if not good:
                ok = False
        h = self._amg_cache.get("P")
        if h is not None:
            for tag, infos in report:
                if tag.startswith("pressure") and infos:
                    h.note_iterations(max(i.innerIterations or i.usedIterations for i in infos))
        for k, tag, (ctas, e0, e1) in self._tuning:
            infos = report[k][1]
            its = max((i.innerIterations or i.usedIterations for i in infos), default=0)
            self.solver_tuner.record(tag, ctas, e0.elapsed_time(e1), its)
        self._tuning.clear()
        self._pending.clear()
        self._last_report = report
        if not ok and raise_on_failure:
            bad = [(t, [str(i) for i in infos if not i.converged]) for t, infos in report]
            raise LinsolveError(f"linear solve failed: {bad}", tag="step")
        return ok

    def _accept_best(self, info: LinearSolverResultInfo) -> bool:
        return False

    def solve_report(self) -> list[tuple[str, list[LinearSolverResultInfo]]]:
        return list(self._last_report)

    def _check_flux_balance(self) -> None:
        d = self.domain
        if d._version == self._flux_checked_version:
            return
        if any(isinstance(b, FixedBoundary) for blk in d.getBlocks() for b in blk.getBoundaries()):
            bal = d.GetBoundaryFluxBalance()
            if float(bal.abs().max()) > float(self.flux_balance_tol):
                raise RuntimeError(
                    f"Domain boundary fluxes not balanced, cannot proceed with simulation step. "
                    f"Flux balance: {bal}, flux_balance_tol: {self.flux_balance_tol}")
        self._flux_checked_version = d._version

    # --- the step ----------------------------------------------------------------------
    def single_step(self, static: bool = False) -> bool:
        """One simulation step of ``substeps`` PISO steps (simulation/simulation.py:262-333)."""
        self._check_flux_balance()
        try:
            if self.substeps == "ADAPTIVE":
                return self._PISO_adaptive_step()
            return self._PISO_split_step(self.substeps)
        except LinsolveError as e:
            self.last_error = str(e)
            return False

    def run(self, iterations: int) -> bool:
        for _ in range(int(iterations)):
            if not self.single_step():
                return False
        return True

    def _PISO_split_step(self, iterations: int, time_step=None) -> bool:
        if not self.differentiable:
            return self._PISO_split_step_plain(iterations, time_step)
        if self._diff is None:
            from .differentiable import DiffRunner

            self._diff = DiffRunner(self)
        if self._nonortho_flags():
            raise NotImplementedError("the differentiable step is the orthogonal step: this grid has cross terms")
        ts = self._time_step_tensor(time_step)
        for _ in range(int(iterations)):
            try:
                self._diff.step(ts)
            except RuntimeError as e:
                self.last_error = str(e)
                return False
        return True

    def detach(self) -> None:
        """Drop the autograd history the simulation keeps between steps (u x e_b of MHD)."""
        if self._diff is not None:
            self._diff.uxb_ag = None

    def _PISO_split_step_plain(self, iterations: int, time_step=None) -> bool:
        d = self.domain
        rec = self._diff if (self._diff is not None and self._diff.rec is not None) else None
        ts = self._time_step_tensor(time_step)
        dims = d.getSpatialDims()
        for step in range(int(iterations)):
            if self.convergence_tol is not None:
                last_vel = d._u_block.clone()
            self._run_hooks(Hook.PRE, local_step=step, time_step=ts)
            flags = self._nonortho_flags()
            matrix_for_velocity = False
            if self.advect_passive_scalar and d.hasPassiveScalar():
                matrix_for_velocity = self._advect_scalar(ts, step, flags)
                if rec is not None:
                    rec.rec.velocity_uses_scalar_matrix = matrix_for_velocity
            self._run_hooks(Hook.PRE_VELOCITY_SETUP, local_step=step, time_step=ts)
            if rec is not None:
                rec.source_in()
            if not matrix_for_velocity:
                backend.SetupAdvectionMatrix(d, ts, flags)
            if not flags:
                backend.SetupAdvectionVelocity(d, ts, 0, False)
                self._run_hooks(Hook.POST_VELOCITY_SETUP, local_step=step, time_step=ts, no_step=0)
                self.solve("C", d.velocityRHS, d.velocityResult, use_BiCG=self.advection_use_BiCG,
                           tol=self.advection_tol, tag="velocity", nrhs=dims)
            else:
                # core/piso_simulation.py:3839-3891: the right-hand side carries the cross terms
                # of the current result, starting from the block velocity; the first solve
                # starts from zero, later ones from the previous result
                backend.CopyVelocityResultFromBlocks(d)
                for no_step in range(self.advect_non_ortho_steps):
                    backend.SetupAdvectionVelocity(d, ts, flags, False)
                    self._run_hooks(Hook.POST_VELOCITY_SETUP, local_step=step, time_step=ts, no_step=no_step)
                    if no_step == 0:
                        d.velocityResult.zero_()
                    self.solve("C", d.velocityRHS, d.velocityResult, use_BiCG=self.advection_use_BiCG,
                               tol=self.advection_tol, tag="velocity", nrhs=dims)
            self._run_hooks(Hook.POST_PREDICTION, local_step=step, time_step=ts)
            for cstep in range(self.corrector_steps):
                if cstep == 0:
                    # P depends on A and the metrics only, so every corrector of a step would
                    # rebuild the same values (pressure.cu:882-927 rebuilds it each time)
                    backend.SetupPressureMatrix(d, ts, flags, False)
                # with flags, the divergence carries the cross terms of the pressure result in
                # place (the previous corrector's), core/piso_simulation.py:3978-4117
                if rec is not None:
                    rec.ustar(d.velocityResult)
                backend.SetupPressureRHS(d, ts, flags, False, False)
                if rec is not None:
                    rec.hbya(d.pressureRHS)
                self._run_hooks(Hook.POST_PRESSURE_SETUP, local_step=step, time_step=ts)
                ex = None
                if self.extrapolate_guesses:
                    ex = self._pressure_extrap.get(cstep)
                    if ex is None:
                        ex = self._pressure_extrap[cstep] = self._new_guess()
                guess = self._pressure_guess.get(cstep) if self.pressure_warm_start else None
                if ex is not None:
                    if not ex.guess(d.pressureResult, d._stencil("P"), d.pressureRHSdiv, d):
                        d.pressureResult.zero_()
                elif guess is not None:
                    d.pressureResult.copy_(guess)
                else:
                    d.pressureResult.zero_()
                self.solve("P", d.pressureRHSdiv, d.pressureResult, use_BiCG=self.pressure_use_BiCG,
                           tol=self._pressure_tol_for(cstep), tag=f"pressure{cstep}",
                           return_best=self.pressure_return_best_result)
                if self.normalize_pressure_result:
                    d._subtract_mean(d.pressureResult, 1)
                if rec is not None:
                    rec.pressure(d.pressureResult)
                for pstep in range(1, self.pressure_non_ortho_steps if flags else 1):
                    # the divergence of the same HbyA with the cross terms of the new result,
                    # re-solved from it
                    backend.SetupPressureRHSdiv(d, ts, flags, False, False)
                    self._run_hooks(Hook.POST_PRESSURE_SETUP, local_step=step, time_step=ts)
                    self.solve("P", d.pressureRHSdiv, d.pressureResult, use_BiCG=self.pressure_use_BiCG,
                               tol=self._pressure_tol_for(cstep), tag=f"pressure{cstep}",
                               return_best=self.pressure_return_best_result)
                    if self.normalize_pressure_result:
                        d._subtract_mean(d.pressureResult, 1)
                if ex is not None:
                    ex.update(d.pressureResult)
                if self.pressure_warm_start:
                    g = self._pressure_guess.get(cstep)
                    if g is None:
                        self._pressure_guess[cstep] = d.pressureResult.clone()
                    else:
                        g.copy_(d.pressureResult)
                self._run_hooks(Hook.POST_PRESSURE_RESULT, local_step=step, time_step=ts)
                backend.CopyPressureResultToBlocks(d)
                backend.CorrectVelocity(d, ts, version=1)
                self._run_hooks(Hook.POST_VELOCITY_CORRECTION, local_step=step, time_step=ts)
            backend.CopyVelocityResultToBlocks(d)
            self._run_hooks(Hook.POST, local_step=step, time_step=ts)
            ok = self.collect_solves() if self.check_solves else True
            self.total_step += 1
            self.total_time += float(ts[0])
            if self.convergence_tol is not None:
                diff = float((last_vel - d._u_block).abs().max())
                if diff < self.convergence_tol:
                    return False
            if not ok:
                return False
        return True

    # --- adaptive substeps (core/piso_simulation.py:4171-4340) -------------------------------
    def _env_state_extras(self) -> list:
        """Getters of per-environment state outside the domain, restored with it for
        environments that sit out a substep."""
        return []

    def _PISO_adaptive_step(self, CFL_cond: float | None = None, max_substeps: int = 1000) -> bool:
        """Advance by `time_step` in substeps that keep the computational-space CFL number
        below `adaptive_CFL`; the substep size is re-derived from the current maximum velocity
        before every substep. Batched domains split per environment (adaptive_CFL_per_env)."""
        d = self.domain
        CFL = self.adaptive_CFL if CFL_cond is None else float(CFL_cond)
        if d.getBatchSize() > 1 and self.adaptive_CFL_per_env:
            if self.differentiable:
                raise NotImplementedError("a differentiable batch takes shared substeps: set adaptive_CFL_per_env=False")
            return self._PISO_adaptive_step_per_env(CFL, max_substeps)
        remaining = self.time_step
        self.adaptive_substeps = 0
        while remaining > 0 and not np.isclose(remaining, 0):
            max_vel = d.getMaxVelocity(True, True).detach().cpu().numpy()
            ts, _ = _cfl_substep(remaining, max_vel, CFL)
            remaining -= ts
            ok = self._PISO_split_step(1, time_step=torch.tensor([float(ts)], dtype=torch.float64))
            self.adaptive_substeps += 1
            if not ok:
                return False
        return True

    def _PISO_adaptive_step_per_env(self, CFL: float, max_substeps: int) -> bool:
        """Every environment splits `time_step` by its own maximum velocity, exactly as it
        would alone; the batch runs until the environment with the most substeps is done, and
        an environment that is done runs the remaining substeps at its last substep size with
        its state restored afterwards (EnvStateSnapshot). Hooks see the [B] substep sizes."""
        from .batching import EnvStateSnapshot

        d = self.domain
        B = d.getBatchSize()
        start = self.total_time
        remaining = [self.time_step] * B
        steps = [self.time_step] * B
        self.adaptive_substeps_per_env = [0] * B
        while True:
            active = [r > 0 and not np.isclose(r, 0) for r in remaining]
            if not any(active):
                break
            mv = d.getMaxVelocityPerEnv(True, True).detach().cpu().numpy()
            for b in range(B):
                if not active[b]:
                    continue
                steps[b], _ = _cfl_substep(remaining[b], mv[b], CFL)
                remaining[b] -= steps[b]
                self.adaptive_substeps_per_env[b] += 1
            done = [b for b in range(B) if not active[b]]
            snap = EnvStateSnapshot(d, torch.tensor(done), extra=self._env_state_extras()) if done else None
            ok = self._PISO_split_step(1, time_step=torch.tensor([float(t) for t in steps], dtype=torch.float64))
            if snap is not None:
                snap.restore()
            self.total_time = start + self.time_step - float(min(remaining))
            if not ok:
                return False
        self.total_time = start + self.time_step
        return True

    def _advect_scalar(self, ts, step: int, flags: int = 0) -> bool:
        """Implicit advection-diffusion of every passive-scalar channel with the velocity of
        the step start (core/piso_simulation.py:3225-3345, 3589-3775): one matrix for all
        channels when their diffusivity and face types agree, else one per channel; a zero
        initial guess; with non-orthogonal flags the right-hand side carries the cross terms
        of the current scalar result and the solve repeats advect_non_ortho_steps times from
        the previous result; the result copied to the blocks. Returns whether the velocity
        step reuses the scalar matrix (same diffusivity as the velocity, one set of face types
        for all channels), as phiPICT does."""
        d = self.domain
        C = d.getPassiveScalarChannels()
        B = d.getBatchSize()
        split = not (d.isPassiveScalarViscosityStatic() and d.isAllFixedBoundariesPassiveScalarTypeStatic())
        reuse = not (d.hasPassiveScalarViscosity() or d.hasBlockViscosity() or d.hasPassiveScalarBlockViscosity() or split)
        rhs = d.scalarRHS.view(B, C, -1)
        res = d.scalarResult.view(B, C, -1)
        if not split:
            backend.SetupAdvectionMatrix(d, ts, flags, forPassiveScalar=True, passiveScalarChannel=0)
        if flags:
            # the cross terms start from the block scalar (core/piso_simulation.py:3272-3283)
            backend.CopyScalarResultFromBlocks(d)
        for no_step in range(self.advect_non_ortho_steps if flags else 1):
            backend.SetupAdvectionScalar(d, ts, flags)
            self._run_hooks(Hook.POST_SCALAR_SETUP, local_step=step, time_step=ts, no_step=no_step)
            for c in range(C):
                if split:
                    backend.SetupAdvectionMatrix(d, ts, flags, forPassiveScalar=True, passiveScalarChannel=c)
                # channel c of every environment as one flat [B][cells] system (launches are
                # stream-ordered, so a per-channel matrix is consumed before the next overwrites it)
                b = rhs[:, c].contiguous().view(-1)
                x = torch.zeros_like(b) if no_step == 0 else res[:, c].reshape(-1).clone()
                self.solve("C", b, x, use_BiCG=self.advection_use_BiCG, tol=self.advection_tol, tag=f"scalar{c}")
                res[:, c].copy_(x.view(B, -1))
        backend.CopyScalarResultToBlocks(d)
        return reuse

    def make_divergence_free(self, iterations: int = 1, max_iter: int = 1000) -> bool:
        """Project the block velocity onto a divergence-free field with A = 1, dt = 1
        (core/piso_simulation.py:3355-3523)."""
        d = self.domain
        ts = torch.tensor([1.0], dtype=torch.float64)
        d.setTimeStep(ts)
        backend.CopyVelocityResultFromBlocks(d)
        for _ in range(int(iterations)):
            d.A.fill_(1.0)
            backend.SetupPressureMatrix(d, ts, 0, False)
            # with A = 1 the projection's HbyA is the velocity itself
            d.pressureRHS.copy_(d.velocityResult)
            backend.SetupPressureRHSdiv(d, ts)
            d.pressureResult.zero_()
            self.solve("P", d.pressureRHSdiv, d.pressureResult, use_BiCG=self.pressure_use_BiCG,
                       tol=self.pressure_tol, tag="projection", max_iter=max_iter)
            if self.normalize_pressure_result:
                d._subtract_mean(d.pressureResult, 1)
            backend.CopyPressureResultToBlocks(d)
            backend.CorrectVelocity(d, ts, version=1)
        backend.CopyVelocityResultToBlocks(d)
        return self.collect_solves(raise_on_failure=False)


def _cfl_substep(time_step_target, max_vel, CFL_cond: float):
    """The next substep size and the number of substeps the remaining time is split into
    (core/piso_simulation.py:187-216): max step CFL / max_vel; NumPy scalars keep their dtype."""
    if np.isclose(max_vel, 0):
        max_time_step = time_step_target
    else:
        max_time_step = CFL_cond / max_vel
    if max_time_step >= time_step_target:
        return time_step_target, 1
    substeps = int(np.ceil(time_step_target / max_time_step))
    return time_step_target / substeps, substeps


def get_max_time_step(domain: Domain, time_step_target: float, CFL_cond: float = 0.8, with_transformations: bool = True):
    """Split a time step into substeps that satisfy a CFL condition (core/piso_simulation.py:
    149-184): returns (substep size, number of substeps)."""
    max_vel = domain.getMaxVelocity(True, with_transformations).cpu().numpy()
    max_time_step = CFL_cond / max_vel
    if max_time_step >= time_step_target:
        return time_step_target, 1
    ss = int(np.ceil(time_step_target / max_time_step))
    return time_step_target / ss, ss
