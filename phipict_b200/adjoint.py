"""Hand-written adjoint of the MHD PISO step with checkpointing, behind torch.autograd.

phiPICT differentiates its step with per-kernel *Grad kernels and an autograd
LinearSolveFunction (core/piso_diff.py:655-1421). Here the reverse pass is the exact
discrete adjoint of the forward kernels, step by step in reverse:

  forward step (FP64; the velocity source is the Lorentz force of this step only):
    S   = N Lor(phi, uxb)                       kCurrentLorentz
    C   = C(u), A = diag C                      kAdvectionMatrix
    u*0 = C^-1 (u/dt + B(u_b)/det + S)          BiCGStab
    P   = P(A)                                  kLaplaceMatrix
    k = 0, 1:  h_k = HbyA(u, u*_k, C, A, S, u_b);  p_k = Pi P^+ div(h_k, u_b)
               u*_{k+1} = h_k - grad(p_k)/A
    u'  = u*_2;  uxb' = u' x e_b;  phi' = Pi E^+ Pi div_E(uxb')

  reverse: the transposed potential solve (CG), the adjoints of the correctors (kernel
  adjoints of the correction, divergence and HbyA, the transposed pressure solves and
  -lambda p^T for the pressure matrix), the transposed momentum solve (BiCGStab on C^T
  built on the device, -lambda u*^T for C), the right-hand side, the advection matrix
  through the face fluxes and the Lorentz force. Pi is the mean projection of the
  rank-deficient systems.

The rollout stores (u, phi, u x e_b) every `checkpoint_every` steps and recomputes each
segment's intermediates during the reverse pass, so memory grows with the segment, not
with the rollout. Gradients are taken with respect to a boundary velocity profile applied
to chosen fixed faces and with respect to the Stuart number of each instance.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass

import torch

from . import _C as backend
from . import _lib
from .mhd import epot_matrix_is_anchored
from .solvers import BICGSTAB, CG, solver_for
from .tolerance import SolverTolerance


@dataclass
class _Record:
    u_in: torch.Tensor
    phi_in: torch.Tensor
    uxb_in: torch.Tensor
    ustar: list
    h: list
    p: list


class AdjointMHD:
    """Forward rollout and reverse pass of ``steps`` MHD PISO steps on a float64 domain.

    faces: (block, face) pairs whose fixed velocity is set to the profile parameter (a
    tensor with the shape of those faces' velocity data, e.g. an inflow and the matching
    outflow of a duct); stuart: [B] Stuart numbers; e_b: (3,) or (B, 3)."""

    def __init__(self, domain, dt: float, stuart: torch.Tensor, e_b: torch.Tensor, steps: int, faces,
                 checkpoint_every: int = 10, tol: float = 1e-13, corrector_steps: int = 2, maxit: int = 20000,
                 mixed_precision: bool = False):
        """mixed_precision: every forward and adjoint solve runs FP32 Krylov iterations
        (multigrid-preconditioned for the pressure and potential systems) inside FP64
        refinement to the same tolerance; the adjoint kernels stay FP64."""
        if domain.getDtype() != torch.float64:
            raise TypeError("the adjoint step runs in float64")
        if not domain.IsInitialized():
            domain.PrepareSolve()
        if domain.getSpatialDims() > 1 and domain.hasNonOrthogonalMetrics():
            raise NotImplementedError("the hand-written adjoint differentiates the orthogonal step; this grid has "
                                      "non-orthogonal cross terms")
        self.d = domain
        self.dims = domain.getSpatialDims()
        self.dt = float(dt)
        self.steps = int(steps)
        self.every = max(1, int(checkpoint_every))
        self.tol = SolverTolerance(rtol=tol)
        self.correctors = int(corrector_steps)
        self.maxit = int(maxit)
        B = domain.getBatchSize()
        dev = domain.getDevice()
        eb = e_b.reshape(1, 3).expand(B, 3) if e_b.dim() == 1 else e_b
        self.e_b = eb.detach().to(dev, torch.float64).contiguous()
        self.stuart = torch.as_tensor(stuart, dtype=torch.float64).reshape(-1).expand(B).contiguous().to(dev)
        self.faces = [domain.getBlock(b).getBoundary(f) if isinstance(b, int) else b.getBoundary(f) for b, f in faces]
        for bd in self.faces:
            if bd._velocity.shape != self.faces[0]._velocity.shape:
                raise ValueError("the parameter faces must share one velocity shape")
        if domain._epot_on is False or getattr(domain, "_E_st", None) is None:
            domain.SetupEpotOnDomain()
        self.rank_deficient_phi = not epot_matrix_is_anchored(domain)
        n = domain.numCells()
        self.uxb = torch.zeros(3 * n, dtype=torch.float64, device=dev)
        self._ts = torch.tensor([self.dt], dtype=torch.float64)
        self.stream = _lib.stream_ptr(dev)
        self.mixed = bool(mixed_precision)
        self._amg_cache: dict = {}
        if self.mixed:
            domain._mixed = True

    # --- state ------------------------------------------------------------------------------
    def _state(self):
        d = self.d
        return d._u_block.reshape(-1).clone(), d.epotResult.clone(), self.uxb.clone()

    def _set_state(self, u, phi, uxb):
        d = self.d
        d._u_block.view(-1).copy_(u)
        d.velocityResult.copy_(u)
        d.epotResult.copy_(phi)
        d._epot_block.view(-1).copy_(phi)
        self.uxb.copy_(uxb)

    def set_profile(self, profile: torch.Tensor) -> None:
        for bd in self.faces:
            bd._velocity.copy_(profile.reshape(bd._velocity.shape))

    # --- one forward step ---------------------------------------------------------------------
    def _solve(self, which, rhs, x, kind, nrhs, A=None):
        d = self.d
        M = d._stencil(which) if A is None else A
        if self.mixed:
            from .amg import hierarchy_for
            from .solvers import refiner_for

            lo = backend._lo(d, which) if A is None else A.float()
            amg = None
            if A is None and kind == CG and nrhs == 1:
                try:
                    amg = hierarchy_for(d, which, lo, d._matrix_version(which), self._amg_cache)
                except ValueError:
                    amg = None
            s = refiner_for(d, kind, nrhs, tag=f"adjoint-{which}-{kind}-{nrhs}", max_outer=30)
            s.solve(M, lo, rhs, x, self.tol, self.maxit, amg=amg)
        else:
            s = solver_for(d, kind, torch.float64, nrhs, tag=f"adjoint-{which}-{kind}-{nrhs}")
            s.solve(M, rhs, x, self.tol, self.maxit)
        bad = [str(i) for i in s.results() if not i.converged]
        if bad:
            raise RuntimeError(f"adjoint rollout: {which} solve did not converge: {bad}")

    def _step(self, record: bool):
        d, lib, st = self.d, _lib.load(), self.stream
        desc = ct.byref(d.desc())
        rec = _Record(*self._state(), [], [], []) if record else None
        d._ensure_cell_source()
        _lib.call("phb_current_lorentz", desc, d.epotResult.data_ptr(), self.uxb.data_ptr(), self.e_b.data_ptr(),
                  self.stuart.data_ptr(), None, d._src.data_ptr(), 0, st)
        backend.SetupAdvectionMatrix(d, self._ts, 0)
        backend.SetupAdvectionVelocity(d, self._ts, 0, False)
        self._solve("C", d.velocityRHS, d.velocityResult, BICGSTAB, self.dims)
        backend.SetupPressureMatrix(d, self._ts, 0, False)
        for _ in range(self.correctors):
            if record:
                rec.ustar.append(d.velocityResult.clone())
            backend.SetupPressureRHS(d, self._ts, 0, False, False)
            d.pressureResult.zero_()
            self._solve("P", d.pressureRHSdiv, d.pressureResult, CG, 1)
            d._subtract_mean(d.pressureResult, 1)
            if record:
                rec.h.append(d.pressureRHS.clone())
                rec.p.append(d.pressureResult.clone())
            backend.CopyPressureResultToBlocks(d)
            backend.CorrectVelocity(d, self._ts, version=1)
        backend.CopyVelocityResultToBlocks(d)
        _lib.call("phb_uxb_epot_rhs", desc, d.velocityResult.data_ptr(), self.e_b.data_ptr(), self.uxb.data_ptr(),
                  d.epotRHS.data_ptr(), st)
        if self.rank_deficient_phi:
            d._subtract_mean(d.epotRHS, 1)
            d._subtract_mean(d.epotResult, 1)
        self._solve("E", d.epotRHS, d.epotResult, CG, 1)
        if self.rank_deficient_phi:
            d._subtract_mean(d.epotResult, 1)
        backend.CopyEpotResultToBlocks(d)
        return rec

    # --- rollout ------------------------------------------------------------------------------
    def forward(self, profile: torch.Tensor | None = None, stuart: torch.Tensor | None = None,
                initial=None) -> torch.Tensor:
        """Run the rollout from `initial` (u, phi, uxb) or the domain's current state; returns
        the final velocity (flat [B][d][cells])."""
        if profile is not None:
            self.set_profile(profile)
        if stuart is not None:
            self.stuart.copy_(torch.as_tensor(stuart, dtype=torch.float64).reshape(-1).expand_as(self.stuart))
        if initial is not None:
            self._set_state(*initial)
        self.checkpoints = []
        for k in range(self.steps):
            if k % self.every == 0:
                self.checkpoints.append(self._state())
            self._step(False)
        return self.d._u_block.reshape(-1).clone()

    # --- reverse --------------------------------------------------------------------------------
    def _zeros(self, n):
        return torch.zeros(n, dtype=torch.float64, device=self.d.getDevice())

    def _proj(self, v):
        w = v.clone()
        self.d._subtract_mean(w, 1)
        return w

    def _step_backward(self, rec: _Record, ubar_out, phibar_out, xbar_out, ubbar, Nbar):
        d, st = self.d, self.stream
        desc = ct.byref(d.desc())
        n, dn = d.numCells(), self.dims * d.numCells()
        S = 2 * self.dims + 1
        # matrices of this step from its input velocity
        d._u_block.view(-1).copy_(rec.u_in)
        backend.SetupAdvectionMatrix(d, self._ts, 0)
        backend.SetupPressureMatrix(d, self._ts, 0, False)
        C, A = d._C_st, d.A
        # potential step
        ubar = ubar_out.clone()
        xbar = xbar_out.clone()
        rhs = self._proj(phibar_out) if self.rank_deficient_phi else phibar_out.clone()
        lam = self._zeros(n)
        self._solve("E", rhs, lam, CG, 1)
        rbar = self._proj(lam) if self.rank_deficient_phi else lam
        _lib.call("phb_adj_uxb_epot_rhs", desc, self.e_b.data_ptr(), rbar.data_ptr(), xbar.data_ptr(), ubar.data_ptr(), st)
        # correctors, last first
        Abar, Cbar, Pbar = self._zeros(n), self._zeros(S * n), self._zeros(S * n)
        Sbar, uin_bar = self._zeros(dn), self._zeros(dn)
        for k in reversed(range(self.correctors)):
            hbar, pbar = self._zeros(dn), self._zeros(n)
            _lib.call("phb_adj_correct_velocity", desc, rec.p[k].data_ptr(), A.data_ptr(), ubar.data_ptr(), hbar.data_ptr(),
                      pbar.data_ptr(), Abar.data_ptr(), st)
            lamP = self._zeros(n)
            self._solve("P", self._proj(pbar), lamP, CG, 1)
            dbar = self._proj(lamP)
            _lib.call("phb_adj_outer", desc, 1, lamP.data_ptr(), rec.p[k].data_ptr(), -1.0, Pbar.data_ptr(), st)
            _lib.call("phb_adj_divergence", desc, dbar.data_ptr(), hbar.data_ptr(), ubbar.data_ptr(), st)
            ustar_bar = self._zeros(dn)
            _lib.call("phb_adj_pressure_rhs", desc, C.data_ptr(), A.data_ptr(), d._u_block.data_ptr(),
                      rec.ustar[k].data_ptr(), rec.h[k].data_ptr(), hbar.data_ptr(), uin_bar.data_ptr(),
                      ustar_bar.data_ptr(), Cbar.data_ptr(), Abar.data_ptr(), Sbar.data_ptr(), ubbar.data_ptr(), st)
            ubar = ustar_bar
        _lib.call("phb_adj_pressure_matrix", desc, A.data_ptr(), Pbar.data_ptr(), Abar.data_ptr(), st)
        # momentum solve on C^T
        CT = torch.empty_like(C)
        _lib.call("phb_transpose_stencil", desc, C.data_ptr(), CT.data_ptr(), st)
        lamM = self._zeros(dn)
        self._solve("C", ubar, lamM, BICGSTAB, self.dims, A=CT)
        _lib.call("phb_adj_outer", desc, self.dims, lamM.data_ptr(), rec.ustar[0].data_ptr(), -1.0, Cbar.data_ptr(), st)
        _lib.call("phb_adj_advection_rhs", desc, lamM.data_ptr(), d._u_block.data_ptr(), uin_bar.data_ptr(),
                  Sbar.data_ptr(), ubbar.data_ptr(), st)
        Cbar.view(S, n)[0] += Abar
        _lib.call("phb_adj_advection_matrix", desc, Cbar.data_ptr(), d._u_block.data_ptr(), uin_bar.data_ptr(), st)
        # Lorentz source
        phi_bar, x_bar = self._zeros(n), self._zeros(3 * n)
        _lib.call("phb_adj_lorentz", desc, rec.phi_in.data_ptr(), rec.uxb_in.data_ptr(), self.e_b.data_ptr(),
                  self.stuart.data_ptr(), Sbar.data_ptr(), phi_bar.data_ptr(), x_bar.data_ptr(), Nbar.data_ptr(), st)
        return uin_bar, phi_bar, x_bar

    def backward(self, ubar_final: torch.Tensor):
        """Gradients of <ubar_final, u_final> with respect to the profile and the Stuart
        numbers (recomputing each checkpoint segment)."""
        d = self.d
        n = d.numCells()
        ubbar = torch.zeros_like(d._fvel)
        Nbar = self._zeros(d.getBatchSize())
        ubar, phibar, xbar = ubar_final.detach().reshape(-1).to(torch.float64).clone(), self._zeros(n), self._zeros(3 * n)
        for seg in reversed(range(len(self.checkpoints))):
            self._set_state(*self.checkpoints[seg])
            first = seg * self.every
            last = min(self.steps, first + self.every)
            recs = [self._step(True) for _ in range(first, last)]
            for rec in reversed(recs):
                ubar, phibar, xbar = self._step_backward(rec, ubar, phibar, xbar, ubbar, Nbar)
        grad_profile = None
        for bd in self.faces:
            off = (bd._velocity.data_ptr() - d._fvel.data_ptr()) // d._fvel.element_size()
            g = ubbar[off:off + bd._velocity.numel()].view(bd._velocity.shape)
            grad_profile = g.clone() if grad_profile is None else grad_profile + g
        return grad_profile, Nbar, ubar


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, profile, stuart, model: AdjointMHD, initial):
        u = model.forward(profile.detach(), stuart.detach(), initial)
        ctx.model = model
        ctx.devices = (profile.device, stuart.device, stuart.shape)
        return u

    @staticmethod
    def backward(ctx, ubar):
        gp, gN, _ = ctx.model.backward(ubar)
        pdev, sdev, sshape = ctx.devices
        if sshape.numel() == 1:
            gN = gN.sum().reshape(sshape)
        return gp.to(pdev), gN.to(sdev).reshape(sshape), None, None


def rollout(model: AdjointMHD, profile: torch.Tensor, stuart: torch.Tensor, initial=None) -> torch.Tensor:
    """Differentiable rollout: the final velocity as a function of the boundary profile and
    the Stuart numbers (torch.autograd)."""
    return _Rollout.apply(profile, stuart, model, initial)


__all__ = ["AdjointMHD", "rollout"]
