"""Differentiable PISO steps behind torch.autograd: ``Simulation(differentiable=True)``.

phiPICT's differentiable backend (core/piso_diff.py, chosen at core/piso_simulation.py:1500)
wraps every stage of the step in a torch.autograd.Function whose backward calls a ``*Grad``
kernel. Here the forward of a step is the ordinary CUDA step, unchanged, while it records
the few intermediates the reverse pass needs (the predictor and corrector velocities, HbyA and
the pressure of every corrector); the backward is the hand-written discrete adjoint of the
whole step (``csrc/adjoint.cu``), one autograd node per step:

  S   = S_in + N Lor(phi_in, uxb_in)      (MHD; the Lorentz force is added onto the source)
  C   = C(u_in), A = diag C
  u*0 = C^-1 rhs(u_in, S, u_b)
  k:    h_k = HbyA(u_in, u*_k, C, A, S, u_b), p_k = Pi P^+ div(h_k, u_b), u*_{k+1} = h_k - grad p_k / A
  u'  = u*_K, p' = p_{K-1};  uxb' = u' x e_b, phi' = Pi E^+ Pi div_E(uxb')   (MHD)

Graph inputs (gradients flow to whichever of them requires grad): the block velocities, the
velocity sources (static [B, d] or per cell), the fixed-face velocities, the Stuart number, the
block potentials. Outputs that carry the graph: the block velocity, pressure and potential, the
velocity source after the Lorentz force, and u x e_b (kept by the simulation for the next step).
Out of scope (refused): grids with non-orthogonal cross terms, the LINEAR_UPWIND scheme, and
per-environment adaptive substeps; passive scalars are transported but not differentiated, and
a hook that replaces the velocity source inside the step cuts the source's gradient there.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field

import torch

from . import _C as backend
from . import _lib
from .solvers import BICGSTAB, CG, solver_for


@dataclass
class StepRecord:
    """Intermediates of one forward step (detached device tensors)."""
    ts: torch.Tensor
    u_in: torch.Tensor
    src_writes: int
    S_in: torch.Tensor | None = None      # source before the Lorentz force (MHD)
    phi_in: torch.Tensor | None = None
    uxb_in: torch.Tensor | None = None
    source_reset: bool = False            # a hook assigned the source during the step
    # the momentum solve reused the passive scalar's matrix (its face types at fixed faces),
    # as phiPICT does when the scalar's diffusivity is the viscosity
    velocity_uses_scalar_matrix: bool = False
    ustar: list = field(default_factory=list)
    h: list = field(default_factory=list)
    p: list = field(default_factory=list)
    phis_in: torch.Tensor | None = None   # passive scalar before and after the step's scalar stage
    phis_out: torch.Tensor | None = None


def _zeros(d, n):
    return torch.zeros(n, dtype=torch.float64, device=d.getDevice())


def _proj(d, v):
    w = v.clone()
    d._subtract_mean(w, 1)
    return w


def adjoint_solve(sim, which: str, rhs: torch.Tensor, x: torch.Tensor, kind: int, nrhs: int, tol, A=None) -> None:
    """A transposed solve of the reverse pass with the simulation's solver settings (FP64
    Krylov, or FP32 Krylov with the multigrid preconditioner inside FP64 refinement)."""
    d = sim.domain
    M = d._stencil(which) if A is None else A
    if sim.mixed_precision:
        from .amg import hierarchy_for
        from .solvers import refiner_for

        lo = backend._lo(d, which) if A is None else A.float()
        amg = None
        if A is None and kind == CG and nrhs == 1 and sim._amg_wanted(which):
            try:
                amg = hierarchy_for(d, which, lo, d._matrix_version(which), sim._amg_cache, sim._amg_options(which))
            except ValueError:
                amg = None
        s = refiner_for(d, kind, nrhs, tag=f"adjoint-{which}-{kind}-{nrhs}", max_outer=30)
        s.solve(M, lo, rhs, x, tol, sim.linear_solve_max_iterations, amg=amg)
    else:
        s = solver_for(d, kind, torch.float64, nrhs, tag=f"adjoint-{which}-{kind}-{nrhs}")
        s.solve(M, rhs, x, tol, sim.linear_solve_max_iterations)
    bad = [str(i) for i in s.results() if not i.converged]
    if bad:
        raise RuntimeError(f"adjoint step: {which} solve did not converge: {bad}")


def viscosity_cotangent(d, rec: StepRecord, Cbar: torch.Tensor, rhsbar: torch.Tensor, nubar: torch.Tensor) -> None:
    """nubar[b] += <Cbar, dC/dnu> + <rhsbar, drhs/dnu> over instance b's cells. The momentum
    matrix and right-hand side are affine in the viscosity (the diffusion coefficients and the
    wall terms 2 nu alpha u_b, advection.cu:27-305,800-954), so their derivatives are exactly
    the differences of the forward kernels run with nu = 1 and nu = 0 at the step's input
    velocity (the source, independent of nu, is left out of both)."""
    st = _lib.stream_ptr(d.getDevice())
    desc = ct.byref(d.desc())
    B, n = d.getBatchSize(), d.numCells()
    dims = d.getSpatialDims()
    S = 2 * dims + 1
    saved = d._nu_dev.clone()
    C1, C0 = torch.empty_like(d._C_st), torch.empty_like(d._C_st)
    A1, A0 = torch.empty_like(d.A), torch.empty_like(d.A)
    r1, r0 = torch.empty_like(d.velocityRHS), torch.empty_like(d.velocityRHS)
    d._u_block.view(-1).copy_(rec.u_in)
    sc = d._scalar_struct() if rec.velocity_uses_scalar_matrix else None
    try:
        for val, C, A, r in ((1.0, C1, A1, r1), (0.0, C0, A0, r0)):
            d._nu_dev.fill_(val)
            if sc is not None:
                _lib.call("phb_scalar_matrix", desc, d._u_block.data_ptr(), ct.byref(sc), 0, C.data_ptr(), A.data_ptr(),
                          None, st)
            else:
                _lib.call("phb_advection_matrix", desc, d._u_block.data_ptr(), C.data_ptr(), A.data_ptr(), None, st)
            _lib.call("phb_advection_rhs", desc, d._u_block.data_ptr(), None, 0, r.data_ptr(), st)
    finally:
        d._nu_dev.copy_(saved)
    per_cell = (Cbar.view(S, n) * (C1 - C0).view(S, n)).sum(0)
    per_cell += (rhsbar.view(B, dims, -1) * (r1 - r0).view(B, dims, -1)).sum(1).reshape(-1)
    nubar += per_cell.view(B, -1).sum(1)


def hbya_viscosity_cotangent(d, rec: StepRecord, k: int, C: torch.Tensor, A: torch.Tensor, hbar: torch.Tensor,
                             nubar: torch.Tensor) -> None:
    """nubar[b] += <hbar, dHbyA/dnu> for corrector k through HbyA's explicit boundary terms
    (pressure.cu:350-521: the fixed faces' 2 nu alpha u_b); its dependence through C and A is
    carried by Cbar and Abar. HbyA is affine in nu at fixed C, A and velocities, so the
    derivative is the difference of the forward kernel run with nu = 1 and nu = 0."""
    st = _lib.stream_ptr(d.getDevice())
    desc = ct.byref(d.desc())
    B, dims = d.getBatchSize(), d.getSpatialDims()
    saved = d._nu_dev.clone()
    h1, h0 = torch.empty_like(rec.h[k]), torch.empty_like(rec.h[k])
    try:
        for val, h in ((1.0, h1), (0.0, h0)):
            d._nu_dev.fill_(val)
            _lib.call("phb_pressure_rhs", desc, C.data_ptr(), A.data_ptr(), rec.u_in.data_ptr(), rec.ustar[k].data_ptr(),
                      None, 0, h.data_ptr(), st)
    finally:
        d._nu_dev.copy_(saved)
    nubar += (hbar.view(B, dims, -1) * (h1 - h0).view(B, dims, -1)).sum((1, 2))


def step_backward(sim, rec: StepRecord, ubar_out, pbar_out, phibar_out, xbar_out, Sbar_out, ubbar, Nbar, mhd: bool,
                  nubar: torch.Tensor | None = None):
    """Reverse pass of one recorded step. Takes the cotangents of the step's outputs (u', p',
    phi', uxb', S; any may be None) and returns those of (u_in, S_in, phi_in, uxb_in); the
    fixed-face and Stuart-number cotangents are accumulated into ubbar and Nbar, and, when
    nubar is given, the viscosity's per instance into nubar."""
    d = sim.domain
    st = _lib.stream_ptr(d.getDevice())
    desc = ct.byref(d.desc())
    B, n, dims = d.getBatchSize(), d.numCells(), d.getSpatialDims()
    dn, S = dims * n, 2 * dims + 1
    ts = rec.ts
    # the matrices of this step, rebuilt from its input velocity
    d._u_block.view(-1).copy_(rec.u_in)
    backend.SetupAdvectionMatrix(d, ts, 0, forPassiveScalar=rec.velocity_uses_scalar_matrix, passiveScalarChannel=0)
    backend.SetupPressureMatrix(d, ts, 0, False)
    C, A = d._C_st, d.A
    ubar = _zeros(d, dn) if ubar_out is None else ubar_out.detach().reshape(-1).to(torch.float64).clone()
    if mhd:
        xbar = _zeros(d, 3 * n) if xbar_out is None else xbar_out.detach().reshape(-1).to(torch.float64).clone()
        if phibar_out is not None:
            pb_ = phibar_out.detach().reshape(-1).to(torch.float64)
            rhs = _proj(d, pb_) if sim._potential_rank_deficient else pb_.clone()
            lam = _zeros(d, n)
            adjoint_solve(sim, "E", rhs, lam, CG, 1, sim.potential_tol)
            rbar = _proj(d, lam) if sim._potential_rank_deficient else lam
            rptr = rbar.data_ptr()
        else:
            rptr = None
        _lib.call("phb_adj_uxb_epot_rhs", desc, sim._e_b_dev.data_ptr(), rptr, xbar.data_ptr(), ubar.data_ptr(), st)
    Abar, Cbar, Pbar = _zeros(d, n), _zeros(d, S * n), _zeros(d, S * n)
    Sbar, uin_bar = _zeros(d, dn), _zeros(d, dn)
    K = len(rec.p)
    for k in reversed(range(K)):
        hbar, pbar = _zeros(d, dn), _zeros(d, n)
        _lib.call("phb_adj_correct_velocity", desc, rec.p[k].data_ptr(), A.data_ptr(), ubar.data_ptr(), hbar.data_ptr(),
                  pbar.data_ptr(), Abar.data_ptr(), st)
        if k == K - 1 and pbar_out is not None:
            pbar += pbar_out.detach().reshape(-1).to(torch.float64)
        lamP = _zeros(d, n)
        adjoint_solve(sim, "P", _proj(d, pbar), lamP, CG, 1, sim.pressure_tol)
        dbar = _proj(d, lamP)
        _lib.call("phb_adj_outer", desc, 1, lamP.data_ptr(), rec.p[k].data_ptr(), -1.0, Pbar.data_ptr(), st)
        _lib.call("phb_adj_divergence", desc, dbar.data_ptr(), hbar.data_ptr(), ubbar.data_ptr(), st)
        if nubar is not None:
            hbya_viscosity_cotangent(d, rec, k, C, A, hbar, nubar)
        ustar_bar = _zeros(d, dn)
        _lib.call("phb_adj_pressure_rhs", desc, C.data_ptr(), A.data_ptr(), d._u_block.data_ptr(), rec.ustar[k].data_ptr(),
                  rec.h[k].data_ptr(), hbar.data_ptr(), uin_bar.data_ptr(), ustar_bar.data_ptr(),
                  Cbar.data_ptr(), Abar.data_ptr(), Sbar.data_ptr(), ubbar.data_ptr(), st)
        ubar = ustar_bar
    _lib.call("phb_adj_pressure_matrix", desc, A.data_ptr(), Pbar.data_ptr(), Abar.data_ptr(), st)
    CT = torch.empty_like(C)
    _lib.call("phb_transpose_stencil", desc, C.data_ptr(), CT.data_ptr(), st)
    lamM = _zeros(d, dn)
    adjoint_solve(sim, "C", ubar, lamM, BICGSTAB, dims, sim.advection_tol, A=CT)
    _lib.call("phb_adj_outer", desc, dims, lamM.data_ptr(), rec.ustar[0].data_ptr(), -1.0, Cbar.data_ptr(), st)
    _lib.call("phb_adj_advection_rhs", desc, lamM.data_ptr(), d._u_block.data_ptr(), uin_bar.data_ptr(), Sbar.data_ptr(),
              ubbar.data_ptr(), st)
    Cbar.view(S, n)[0] += Abar
    _lib.call("phb_adj_advection_matrix", desc, Cbar.data_ptr(), d._u_block.data_ptr(), uin_bar.data_ptr(), st)
    if nubar is not None:
        viscosity_cotangent(d, rec, Cbar, lamM, nubar)
    if Sbar_out is not None:
        Sbar += Sbar_out.detach().reshape(-1).to(torch.float64)
    phi_bar = x_bar = None
    if mhd:
        phi_bar, x_bar = _zeros(d, n), _zeros(d, 3 * n)
        _lib.call("phb_adj_lorentz", desc, rec.phi_in.data_ptr(), rec.uxb_in.data_ptr(), sim._e_b_dev.data_ptr(),
                  sim._stuart_dev.data_ptr(), Sbar.data_ptr(), phi_bar.data_ptr(), x_bar.data_ptr(), Nbar.data_ptr(), st)
    S_in_bar = None if rec.source_reset else Sbar
    return uin_bar, S_in_bar, phi_bar, x_bar


def scalar_backward(sim, rec: StepRecord, phisbar: torch.Tensor, uin_bar: torch.Tensor, ubbar: torch.Tensor,
                    nubar: torch.Tensor | None):
    """Reverse pass of the step's passive-scalar stage (every channel c solved from zero with
    its advection-diffusion matrix C_c(u_in) and right-hand side r(phi_in, boundary values,
    boundary velocities); advection.cu:27-305,545-698, core/piso_simulation.py:3589-3775):
    lambda_c = C_c^-T phibar_c, then C_c's cotangent -lambda_c phi_c^T -> u_in, and the
    right-hand side's cotangent lambda -> phi_in, the boundary scalar values and velocities.
    The scalar's diffusivity is the velocity's when the domain sets none; then the viscosity's
    cotangent gets the stage's share. Returns (phi_in bar, boundary values bar)."""
    d = sim.domain
    st = _lib.stream_ptr(d.getDevice())
    desc = ct.byref(d.desc())
    B, n = d.getBatchSize(), d.numCells()
    Cn = d.getPassiveScalarChannels()
    dims = d.getSpatialDims()
    S = 2 * dims + 1
    sc = d._scalar_struct()
    d._u_block.view(-1).copy_(rec.u_in)
    phis_out = rec.phis_out.view(B, Cn, -1)
    gout = phisbar.detach().reshape(B, Cn, -1).to(torch.float64)
    rhsbar = torch.zeros(B, Cn, n // B, dtype=torch.float64, device=d.getDevice())
    split = not (d.isPassiveScalarViscosityStatic() and d.isAllFixedBoundariesPassiveScalarTypeStatic())
    nu_shared = sc.nu_count == 0
    for c in range(Cn):
        if c == 0 or split:
            backend.SetupAdvectionMatrix(d, rec.ts, 0, forPassiveScalar=True, passiveScalarChannel=c)
            CT = torch.empty_like(d._C_st)
            _lib.call("phb_transpose_stencil", desc, d._C_st.data_ptr(), CT.data_ptr(), st)
            Cs = d._C_st.clone()
        g = gout[:, c].contiguous().view(-1)
        if not bool(g.any()):
            continue
        lam = _zeros(d, n)
        adjoint_solve(sim, "C", g, lam, BICGSTAB, 1, sim.advection_tol, A=CT)
        rhsbar[:, c] = lam.view(B, -1)
        Cbar = _zeros(d, S * n)
        x = phis_out[:, c].contiguous().view(-1)
        _lib.call("phb_adj_outer", desc, 1, lam.data_ptr(), x.data_ptr(), -1.0, Cbar.data_ptr(), st)
        _lib.call("phb_adj_advection_matrix", desc, Cbar.data_ptr(), d._u_block.data_ptr(), uin_bar.data_ptr(), st)
        if nubar is not None and nu_shared:
            saved = d._nu_dev.clone()
            C1, C0 = torch.empty_like(Cs), torch.empty_like(Cs)
            A1, A0 = torch.empty_like(d.A), torch.empty_like(d.A)
            try:
                for val, Cv, Av in ((1.0, C1, A1), (0.0, C0, A0)):
                    d._nu_dev.fill_(val)
                    _lib.call("phb_scalar_matrix", desc, d._u_block.data_ptr(), ct.byref(sc), c, Cv.data_ptr(),
                              Av.data_ptr(), None, st)
            finally:
                d._nu_dev.copy_(saved)
            nubar += (Cbar.view(S, n) * (C1 - C0).view(S, n)).sum(0).view(B, -1).sum(1)
    phis_in = rec.phis_in
    phis_in_bar = torch.zeros_like(phis_in)
    fscal_bar = torch.zeros_like(d._fscal, dtype=torch.float64)
    _lib.call("phb_adj_scalar_rhs", desc, ct.byref(sc), phis_in.data_ptr(), d._u_block.data_ptr(), rhsbar.data_ptr(),
              phis_in_bar.data_ptr(), fscal_bar.data_ptr(), uin_bar.data_ptr(), ubbar.data_ptr(), st)
    if nubar is not None and nu_shared:
        saved = d._nu_dev.clone()
        r1, r0 = torch.empty_like(rhsbar), torch.empty_like(rhsbar)
        try:
            for val, r in ((1.0, r1), (0.0, r0)):
                d._nu_dev.fill_(val)
                _lib.call("phb_scalar_rhs", desc, phis_in.data_ptr(), d._u_block.data_ptr(), ct.byref(sc), r.data_ptr(), st)
        finally:
            d._nu_dev.copy_(saved)
        nubar += (rhsbar * (r1 - r0)).sum((1, 2))
    return phis_in_bar, fscal_bar


class _DiffStep(torch.autograd.Function):
    """One PISO step as one autograd node (forward: the CUDA step; backward: its adjoint)."""

    @staticmethod
    def forward(ctx, runner, u_in, S_in, fvel, stuart, phi_in, uxb_in, nu, phis_in, fscal):
        outs, rec = runner.forward_step()
        ctx.runner, ctx.rec = runner, rec
        ctx.shapes = (u_in.shape, S_in.shape, fvel.shape, stuart.shape, phi_in.shape, uxb_in.shape)
        ctx.stuart_device = stuart.device
        ctx.nu_shape, ctx.nu_device = nu.shape, nu.device
        ctx.scalar_shapes = (phis_in.shape, fscal.shape)
        return outs

    @staticmethod
    def backward(ctx, ubar, pbar, phibar, xbar, Sbar, phisbar):
        runner, rec = ctx.runner, ctx.rec
        sim = runner.sim
        d = sim.domain
        ubbar = torch.zeros_like(d._fvel, dtype=torch.float64)
        Nbar = torch.zeros(d.getBatchSize(), dtype=torch.float64, device=d.getDevice())
        nubar = torch.zeros(d.getBatchSize(), dtype=torch.float64, device=d.getDevice()) \
            if ctx.needs_input_grad[7] else None
        state = runner.save_state()
        g_phis = g_fscal = None
        try:
            uin_bar, S_bar, phi_bar, x_bar = step_backward(sim, rec, ubar, pbar, phibar if runner.mhd else None,
                                                          xbar if runner.mhd else None, Sbar, ubbar, Nbar, runner.mhd,
                                                          nubar)
            if runner.scalar and phisbar is not None:
                g_phis, g_fscal = scalar_backward(sim, rec, phisbar, uin_bar, ubbar, nubar)
                g_phis = g_phis.view(ctx.scalar_shapes[0])
                g_fscal = g_fscal.view(ctx.scalar_shapes[1])
        finally:
            runner.restore_state(state)
        g_nu = None
        if nubar is not None:
            g_nu = (nubar.sum() if ctx.nu_shape.numel() == 1 else nubar).reshape(ctx.nu_shape).to(ctx.nu_device)
        su, sS, sf, sN, sp, sx = ctx.shapes
        g_u = uin_bar.view(su)
        g_S = S_bar.view(sS) if S_bar is not None else None
        g_f = ubbar.view(sf)
        g_N = None
        if runner.mhd:
            g_N = (Nbar.sum().reshape(sN) if sN.numel() == 1 else Nbar.reshape(sN)).to(ctx.stuart_device)
        g_p = phi_bar.view(sp) if phi_bar is not None else None
        g_x = x_bar.view(sx) if x_bar is not None else None
        return None, g_u, g_S, g_f, g_N, g_p, g_x, g_nu, g_phis, g_fscal


class DiffRunner:
    """Runs the differentiable steps of a Simulation (set up by ``differentiable=True``)."""

    def __init__(self, sim):
        self.sim = sim
        d = sim.domain
        if d.getDtype() != torch.float64:
            raise TypeError("a differentiable simulation runs on a float64 domain")
        if d.getSpatialDims() > 1 and d.hasNonOrthogonalMetrics() and sim.non_orthogonal:
            raise NotImplementedError("the hand-written adjoint differentiates the orthogonal step; this grid has "
                                      "non-orthogonal cross terms (use non_orthogonal=False only if they vanish)")
        self.mhd = hasattr(sim, "_stuart_number")
        self.scalar = bool(sim.advect_passive_scalar and d.hasPassiveScalar())
        self.rec: StepRecord | None = None
        self.uxb_ag: torch.Tensor | None = None

    # --- recording (called by the Simulation's step) ----------------------------------------
    def begin(self, ts):
        d = self.sim.domain
        self.rec = StepRecord(ts=ts.clone(), u_in=d._u_block.reshape(-1).clone(), src_writes=d._source_writes)
        if self.scalar:
            self.rec.phis_in = d._phi_block.reshape(-1).clone()

    def source_in(self):
        """Just before the Lorentz force is added (MHD) or the momentum is set up."""
        r, d, sim = self.rec, self.sim.domain, self.sim
        if r is None or r.S_in is not None:
            return
        d._ensure_cell_source()
        r.S_in = d._src.reshape(-1).clone()
        r.source_reset = d._source_writes != r.src_writes
        if self.mhd:
            r.phi_in = d.epotResult.clone()
            r.uxb_in = sim._uxb.clone()

    def ustar(self, v):
        if self.rec is not None:
            self.rec.ustar.append(v.clone())

    def hbya(self, h):
        if self.rec is not None:
            self.rec.h.append(h.clone())

    def pressure(self, p):
        if self.rec is not None:
            self.rec.p.append(p.clone())

    # --- state kept across the reverse pass -------------------------------------------------
    def save_state(self):
        d = self.sim.domain
        keep = [d._u_block, d.velocityResult, d.pressureResult, d._p_block, d.A, d._C_st, d._P_st]
        if self.mhd:
            keep += [d.epotResult, d._epot_block, self.sim._uxb]
        if d._src is not None:
            keep.append(d._src)
        if self.scalar:
            keep += [d._phi_block, d.scalarResult, d.scalarRHS]
        return [(t, t.clone()) for t in keep]

    @staticmethod
    def restore_state(state):
        for t, v in state:
            t.copy_(v)

    # --- graph inputs and outputs ------------------------------------------------------------
    def _gather_blocks(self, field_ag: str, field: str, comps: int) -> torch.Tensor:
        d = self.sim.domain
        B = d.getBatchSize()
        parts = []
        for b in d.getBlocks():
            t = getattr(b, field_ag)
            if t is None:
                t = getattr(b, field).detach()
            parts.append(t.reshape(t.shape[0], comps, -1).expand(B, comps, b.ncells()))
        return torch.cat(parts, dim=2)

    def _gather_source(self) -> torch.Tensor:
        d = self.sim.domain
        B, dims = d.getBatchSize(), d.getSpatialDims()
        d._ensure_cell_source()
        if not any(b._source_ag is not None for b in d.getBlocks()):
            return d._src.detach().reshape(B, dims, -1)
        parts = []
        for b in d.getBlocks():
            n = b.ncells()
            s = b._source_ag
            if s is None:
                s = d._block_view(b, "velocitySource").detach()
            s = s.reshape(s.shape[0], dims, 1) if s.dim() == 2 else s.reshape(s.shape[0], dims, n)
            parts.append(s.expand(B, dims, n))
        return torch.cat(parts, dim=2)

    def _gather_fvel(self) -> torch.Tensor:
        d = self.sim.domain
        f = d._fvel.detach()
        fixed = [bd for b in d.getBlocks() for bd in b.getBoundaries() if getattr(bd, "_velocity_ag", None) is not None]
        if not fixed:
            return f
        f = f.clone()
        for bd in fixed:
            off = (bd._velocity.data_ptr() - d._fvel.data_ptr()) // d._fvel.element_size()
            v = bd._velocity_ag.to(torch.float64)
            f[off:off + bd._velocity.numel()] = v.expand(bd._velocity.shape).reshape(-1)
        return f

    def _gather_fscal(self) -> torch.Tensor:
        d = self.sim.domain
        f = d._fscal.detach()
        fixed = [bd for b in d.getBlocks() for bd in b.getBoundaries() if getattr(bd, "_scalar_ag", None) is not None]
        if not fixed:
            return f
        f = f.clone()
        for bd in fixed:
            off = (bd._passiveScalar.data_ptr() - d._fscal.data_ptr()) // d._fscal.element_size()
            v = bd._scalar_ag.to(torch.float64)
            f[off:off + bd._passiveScalar.numel()] = v.expand(bd._passiveScalar.shape).reshape(-1)
        return f

    def step(self, ts) -> None:
        """One recorded step wrapped as a graph node; the block fields become its outputs."""
        sim, d = self.sim, self.sim.domain
        B, dims, N = d.getBatchSize(), d.getSpatialDims(), d.getTotalSize()
        u_in = self._gather_blocks("_velocity_ag", "velocity", dims)
        S_in = self._gather_source()
        fvel = self._gather_fvel()
        if self.mhd:
            st = sim._stuart_number
            stuart = st if isinstance(st, torch.Tensor) else torch.tensor(float(st))
            phi_in = self._gather_blocks("_epot_ag", "epot", 1)
            uxb_in = self.uxb_ag if self.uxb_ag is not None else sim._uxb.detach()
        else:
            stuart = torch.zeros(1, dtype=torch.float64)
            phi_in = torch.zeros(1, dtype=torch.float64, device=d.getDevice())
            uxb_in = torch.zeros(1, dtype=torch.float64, device=d.getDevice())
        nu = d._viscosity_ag if d._viscosity_ag is not None else d.viscosity
        if self.scalar:
            Cn = d.getPassiveScalarChannels()
            phis_in = self._gather_blocks("_scalar_ag", "passiveScalar", Cn)
            fscal = self._gather_fscal()
        else:
            phis_in = torch.zeros(1, dtype=torch.float64, device=d.getDevice())
            fscal = torch.zeros(1, dtype=torch.float64, device=d.getDevice())
        self._ts = ts
        u, p, phi, uxb, S, phis = _DiffStep.apply(self, u_in, S_in, fvel, stuart, phi_in, uxb_in, nu, phis_in, fscal)
        # the block fields become views of the graph outputs (the flat buffers keep the values)
        for b in d.getBlocks():
            o, n = b.globalOffset, b.ncells()
            spatial = list(reversed(b._sizes[:dims]))
            b.velocity = u[:, :, o:o + n].view(B, dims, *spatial)
            b._velocity_ag = b.velocity
            b.pressure = p[:, o:o + n].view(B, 1, *spatial)
            b._pressure_ag = b.pressure
            b.velocitySource = S[:, :, o:o + n].view(B, dims, *spatial)
            b._source_ag = b.velocitySource
            if self.mhd:
                b.epot = phi[:, o:o + n].view(B, 1, *spatial)
                b._epot_ag = b.epot
            if self.scalar:
                b.passiveScalar = phis[:, :, o:o + n].view(B, phis.shape[1], *spatial)
                b._scalar_ag = b.passiveScalar
        self.uxb_ag = uxb if self.mhd else None

    def forward_step(self):
        """The ordinary step with recording; returns the outputs (u, p, phi, uxb, S, passive scalar)
        and the record."""
        sim, d = self.sim, self.sim.domain
        B, dims, N = d.getBatchSize(), d.getSpatialDims(), d.getTotalSize()
        self.begin(self._ts)
        try:
            ok = sim._PISO_split_step_plain(1, self._ts)
        finally:
            rec, self.rec = self.rec, None
        if not ok:
            raise RuntimeError(f"differentiable step failed: {sim.last_error}")
        if rec.S_in is None:  # no Lorentz hook ran (plain PISO): the source as the step used it
            rec.S_in = d._src.reshape(-1).clone()
        if self.scalar:
            rec.phis_out = d._phi_block.reshape(-1).clone()
        zero = torch.zeros(1, dtype=torch.float64, device=d.getDevice())
        outs = (d._u_block.view(B, dims, N).clone(), d.pressureResult.view(B, N).clone(),
                d.epotResult.view(B, N).clone() if self.mhd else zero,
                sim._uxb.clone() if self.mhd else zero.clone(),
                d._src.view(B, dims, N).clone(),
                d._phi_block.view(B, -1, N).clone() if self.scalar else zero.clone())
        return outs, rec


__all__ = ["DiffRunner", "StepRecord", "step_backward"]
