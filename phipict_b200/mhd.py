"""Inductionless (low-Rm) MHD on top of the PISO step (phiPICT simulation/mhd.py).

Governing equations (non-dimensional): ``j = -grad(phi) + u x e_b``,
``laplacian(phi) = div(u x e_b)``, ``F_L = N (j x e_b)`` with ``N = Ha^2/Re``.

As in phiPICT the potential step runs at the POST hook of every PISO step (mhd.py:877-1002)
and the Lorentz force is added to the velocity source at PRE_VELOCITY_SETUP
(mhd.py:543-595), including phiPICT's accumulation onto an existing source. Here both are
single fused kernels: u x e_b with the potential right-hand side, and the face-based current
density with the Lorentz force.
"""
from __future__ import annotations

import torch

from . import _C as backend
from .domain import Domain
from .hooks import Hook, Hooks
from .simulation import Simulation
from .solvers import LinearSolverResultInfo
from .tolerance import SolverTolerance, coerce_tolerance


def epot_matrix_is_anchored(domain: Domain) -> bool:
    """True if a Dirichlet potential face makes the potential matrix non-singular (mhd.py:48-80)."""
    if hasattr(domain, "members"):  # a DomainBatch: its instances must agree
        from .batch import potential_anchoring

        return potential_anchoring(domain)
    for block in domain.getBlocks():
        for _, bound in block.getFixedBoundaries():
            if bound.hasPotentialDirichlet():
                return True
    return False


class MHDSimulation(Simulation):
    """A drop-in for ``phipict.MHDSimulation``.

    ``stuart_number`` may hold one value or one per batched environment; ``e_b`` is a
    uniform field of shape ``(3,)`` or one per environment ``(B, 3)``."""

    def __init__(
        self,
        domain: Domain,
        dt: float,
        stuart_number: torch.Tensor,
        e_b: torch.Tensor,
        potential_tol: float | SolverTolerance | None = None,
        potential_use_BiCG: bool = False,
        potential_normalize: bool = True,
        potential_non_ortho_flags: int = 0,
        potential_use_face_transform: bool = False,
        potential_solve_max_iter: int = 5000,
        potential_solve_dtype: torch.dtype | None = None,
        exclude_potential_solve_gradients: bool = False,
        potential_reuse_result: bool = True,
        potential_return_best_result: bool = True,
        potential_use_preconditioner: bool = False,
        potential_amg_options: dict | None = None,
        **kwargs,
    ) -> None:
        hooks, prep_fn = kwargs.pop("hooks", None), kwargs.pop("prep_fn", None)
        if hooks is not None and prep_fn is not None:
            raise ValueError("Pass hooks or its former name prep_fn, not both.")
        hooks = Hooks(hooks if hooks is not None else prep_fn)
        super().__init__(domain=domain, dt=dt, hooks=hooks, **kwargs)
        if not isinstance(stuart_number, torch.Tensor):
            stuart_number = torch.tensor(float(stuart_number))
        B = domain.getBatchSize()
        if stuart_number.numel() not in (1, B):
            raise ValueError("stuart_number must be a scalar tensor (or one value per environment).")
        if potential_solve_dtype is not None and potential_solve_dtype != domain.getDtype():
            raise NotImplementedError("use mixed_precision=True for a refined potential solve")
        if potential_use_preconditioner:
            from .amg import require_amg

            require_amg()
            if not self._amg_dtype_ok():
                raise NotImplementedError(
                    "the multigrid V-cycle runs in float32: use a float32 domain or mixed_precision=True")
        self._potential_amg_options = dict(potential_amg_options or {})
        self._stuart_number = stuart_number
        self.potential_tol = coerce_tolerance(potential_tol)
        self._potential_use_BiCG = potential_use_BiCG
        self._potential_normalize = potential_normalize
        self._potential_solve_max_iter = int(potential_solve_max_iter)
        self._potential_reuse_result = potential_reuse_result
        self._potential_return_best_result = potential_return_best_result
        self._potential_use_preconditioner = potential_use_preconditioner
        self._dims = domain.getSpatialDims()
        dev = domain.getDevice()
        self._set_field(e_b)
        self._stuart_dev = stuart_number.detach().to(dev, torch.float64).reshape(-1).expand(B).contiguous()
        domain.SetupEpotOnDomain(potential_non_ortho_flags, potential_use_face_transform)
        self._potential_rank_deficient = not epot_matrix_is_anchored(domain)
        # u x e_b of the last potential step, [B][3][cells]; phiPICT initialises it from
        # domain.velocityResult, which is zero until a step has run (mhd.py:526-533)
        self._uxb = torch.zeros(3 * domain.numCells(), dtype=domain.getDtype(), device=dev)
        self._potential_stale = False
        self.hooks.append(Hook.POST, self._magnetic_step_callback)
        self.hooks.append(Hook.PRE_VELOCITY_SETUP, self._add_lorentz_force)

    # potential solves use the multigrid preconditioner when asked (mhd.py:673-712)
    def _amg_wanted(self, which: str) -> bool:
        if which == "E":
            return bool(self._potential_use_preconditioner) and not self._potential_use_BiCG
        return super()._amg_wanted(which)

    def _amg_options(self, which: str) -> dict:
        return self._potential_amg_options if which == "E" else super()._amg_options(which)

    def _set_field(self, e_b: torch.Tensor) -> None:
        d = self.domain
        B = d.getBatchSize()
        if not isinstance(e_b, torch.Tensor):
            raise ValueError("e_b must be a torch.Tensor.")
        if e_b.dim() == 1 and e_b.shape == (3,):
            eb = e_b.reshape(1, 3).expand(B, 3)
        elif e_b.dim() == 2 and e_b.shape == (B, 3):
            eb = e_b
        else:
            raise NotImplementedError("phipict_b200 takes a uniform magnetic field (3,) or one per environment (B, 3)")
        self._e_b = e_b
        self._e_b_dev = eb.detach().to(d.getDevice(), torch.float64).contiguous()

    @property
    def magnetic_field(self) -> torch.Tensor:
        return self._e_b

    @magnetic_field.setter
    def magnetic_field(self, e_b: torch.Tensor) -> None:
        self._set_field(e_b)
        self._potential_stale = False

    def set_magnetic_field(self, e_b: torch.Tensor) -> None:
        old = self._e_b_dev.clone()
        self._set_field(e_b)
        if not torch.equal(old, self._e_b_dev):
            self._potential_stale = True

    def _env_state_extras(self) -> list:
        """Adds u x e_b of the last magnetic step, which the next substep's Lorentz force uses
        (simulation/mhd.py:864-875)."""
        return [*super()._env_state_extras(), lambda: self._uxb]

    def _accept_best(self, info: LinearSolverResultInfo) -> bool:
        # a non-converged plain solve returns its best iterate (mhd.py:430-433); a refined
        # solve has no best iterate, so it has to converge
        return self._potential_return_best_result and info.isFiniteResidual and not self.mixed_precision

    # --- hooks -------------------------------------------------------------------------
    def _add_lorentz_force(self, domain: Domain, **kwargs) -> None:
        """J from phi and u x e_b, F_L = N (J x e_b) added onto the velocity source."""
        if self._diff is not None and self._diff.rec is not None:
            self._diff.source_in()  # the source before the force, for the reverse pass
        if self._potential_stale:
            self._magnetic_step_callback(domain)
            self._potential_stale = False
        had_source = domain._src_mode != 0
        domain._ensure_cell_source()
        import ctypes as ct

        from . import _lib

        _lib.call("phb_current_lorentz", ct.byref(domain.desc()), domain.epotResult.data_ptr(), self._uxb.data_ptr(),
                  self._e_b_dev.data_ptr(), self._stuart_dev.data_ptr(), None, domain._src.data_ptr(),
                  1 if had_source else 0, _lib.stream_ptr(domain.getDevice()))

    def _magnetic_step_callback(self, domain: Domain, time_step=None, max_iter: int | None = None, **kwargs) -> bool:
        """u x e_b, its divergence, and the potential solve (mhd.py:877-1002)."""
        import ctypes as ct

        from . import _lib

        _lib.call("phb_uxb_epot_rhs", ct.byref(domain.desc()), domain.velocityResult.data_ptr(), self._e_b_dev.data_ptr(),
                  self._uxb.data_ptr(), domain.epotRHS.data_ptr(), _lib.stream_ptr(domain.getDevice()))
        if self._potential_rank_deficient:
            domain._subtract_mean(domain.epotRHS, 1)
        if not self._potential_reuse_result:
            domain.epotResult.zero_()
        else:
            ex = None
            if self.extrapolate_guesses:
                ex = self.__dict__.get("_epot_extrap")
                if ex is None:
                    ex = self._epot_extrap = self._new_guess()
                    ex.update(domain.epotResult)  # the current potential is the first result
                ex.guess(domain.epotResult, domain._stencil("E"), domain.epotRHS, domain)
            if self._potential_rank_deficient:
                domain._subtract_mean(domain.epotResult, 1)
        self.solve("E", domain.epotRHS, domain.epotResult, use_BiCG=self._potential_use_BiCG, tol=self.potential_tol,
                   tag="epot", return_best=self._potential_return_best_result,
                   max_iter=self._potential_solve_max_iter if max_iter is None else max_iter)
        if self._potential_reuse_result and self.extrapolate_guesses:
            self._epot_extrap.update(domain.epotResult)
        if self._potential_normalize and self._potential_rank_deficient:
            domain._subtract_mean(domain.epotResult, 1)
        backend.CopyEpotResultToBlocks(domain)
        return True

    def make_current_divergence_free(self, max_iter: int = 1000) -> bool:
        backend.CopyVelocityResultFromBlocks(self.domain)
        self._magnetic_step_callback(self.domain, max_iter=max_iter)
        self._potential_stale = False
        return self.collect_solves(raise_on_failure=False)

    def get_current_density(self, block) -> torch.Tensor:
        """j = -grad(phi) + u x e_b of a block from the face-based reconstruction, [B, 3, *spatial]."""
        d = self.domain
        J = backend.ComputeCurrentDensityFaceBased(d, d.epotResult, self._uxb)
        B, N = d.getBatchSize(), d.getTotalSize()
        n = block.ncells()
        spatial = list(reversed(block.getSizes()[: self._dims]))
        return J.view(B, 3, N)[:, :, block.globalOffset:block.globalOffset + n].reshape(B, 3, *spatial)

    def detach(self) -> None:
        super().detach()
