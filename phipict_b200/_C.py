"""Backend protocol of the PISO step: the functions phiPICT's simulation driver calls on
its ``_C`` module (csrc/phipict/bindings.cpp:639-815), with the same names, arguments and
in-place semantics, implemented on the phipict_b200 CUDA kernels.

Every function launches on torch's current CUDA stream and returns without synchronising
the device (phiPICT's launchers call ``cudaDeviceSynchronize()`` around every kernel,
e.g. piso/advection.cu:1217,1225). Matrices live in stencil form on the domain
(``domain._C_st`` etc.); ``domain.C``/``domain.P``/``domain.Epot`` are CSR views of them.
"""
from __future__ import annotations

import ctypes as ct
import math

import torch

from . import _lib
from .domain import CSRmatrix, Domain
from .solvers import BICGSTAB, CG, LinearSolverResultInfo, solver_for

NON_ORTHO_DIRECT_MATRIX = 1
NON_ORTHO_DIRECT_RHS = 2
NON_ORTHO_DIAGONAL_MATRIX = 4
NON_ORTHO_DIAGONAL_RHS = 8
NON_ORTHO_CENTER_MATRIX = 16


def _check(domain: Domain) -> None:
    if domain.getNumBlocks() == 0:
        raise RuntimeError("Domain does not contain blocks.")
    if not domain.IsInitialized():
        raise RuntimeError("Domain is not initialized.")


NON_ORTHO_RHS = NON_ORTHO_DIRECT_RHS | NON_ORTHO_DIAGONAL_RHS


def _flags(flags) -> int:
    """The non-orthogonal flag bits of one Setup* call (piso/non_ortho_flags.h:23-27)."""
    f = int(flags)
    if not 0 <= f < 32:
        raise ValueError(f"invalid non-orthogonal flags {flags}")
    return f


def _desc(domain: Domain, flags: int = 0) -> _lib.PhbDomain:
    """The domain's descriptor carrying this call's non-orthogonal flags (a copy: the cached
    descriptor keeps 0 for every caller that passes none)."""
    d = domain.desc()
    if not flags:
        return d
    c = _lib.PhbDomain.from_buffer_copy(d)
    c.nonortho = flags
    return c


def _S(domain: Domain) -> int:
    return _lib.stream_ptr(domain.getDevice())


def _lo(domain: Domain, which: str) -> torch.Tensor | None:
    """The float32 shadow of a float64 stencil matrix (mixed precision), if enabled."""
    if not getattr(domain, "_mixed", False):
        return None
    key = "_" + which + "_lo"
    t = getattr(domain, key, None)
    st = domain._stencil(which)
    ver = domain._matrix_version(which)
    lover = domain.__dict__.setdefault("_lo_ver", {})
    if t is None or t.shape != st.shape:
        t = torch.empty(st.shape, dtype=torch.float32, device=st.device)
        setattr(domain, key, t)
        lover[which] = None
    if lover.get(which) != ver:
        # the momentum and pressure kernels refresh their copies at every assembly; the
        # potential matrix (assembled once) and values set through the CSR views are
        # copied here
        t.copy_(st)
        lover[which] = ver
    return t


def _assembled(domain: Domain, which: str, lo: torch.Tensor | None) -> None:
    """A kernel rewrote stencil ``which`` (and its float32 copy ``lo`` when given)."""
    ver = domain._bump_matrix(which)
    if lo is not None:
        domain.__dict__.setdefault("_lo_ver", {})[which] = ver


def _src(domain: Domain) -> tuple[int | None, int]:
    return (domain._src.data_ptr() if domain._src is not None else None), domain._src_mode


# --- momentum ---------------------------------------------------------------------------
def SetupAdvectionMatrix(domain: Domain, timeStep, nonOrthoFlags=0, forPassiveScalar: bool = False,
                         passiveScalarChannel: int = 0) -> None:
    """Implicit Euler advection-diffusion matrix C and its diagonal A (advection.cu:27-305)."""
    _check(domain)
    desc = _desc(domain, _flags(nonOrthoFlags))
    domain.setTimeStep(timeStep)
    lo = _lo(domain, "C")
    if forPassiveScalar:
        c = int(passiveScalarChannel)
        if not 0 <= c < domain.getPassiveScalarChannels():
            raise RuntimeError(f"passive scalar channel {c} out of range")
        _lib.call("phb_scalar_matrix", ct.byref(desc), domain._u_block.data_ptr(), ct.byref(domain._scalar_struct()),
                  c, domain._C_st.data_ptr(), domain.A.data_ptr(), lo.data_ptr() if lo is not None else None, _S(domain))
    else:
        _lib.call("phb_advection_matrix", ct.byref(desc), domain._u_block.data_ptr(), domain._C_st.data_ptr(),
                  domain.A.data_ptr(), lo.data_ptr() if lo is not None else None, _S(domain))
    _assembled(domain, "C", lo)


def SetupAdvectionVelocity(domain: Domain, timeStep, nonOrthoFlags=0, applyPressureGradient: bool = False) -> None:
    """Momentum right-hand side into ``domain.velocityRHS`` (advection.cu:800-954); with
    non-orthogonal right-hand-side flags it carries the cross terms of ``velocityResult``."""
    _check(domain)
    flags = _flags(nonOrthoFlags)
    if applyPressureGradient:
        raise NotImplementedError("applyPressureGradient is not used by the PISO step")
    domain.setTimeStep(timeStep)
    src, mode = _src(domain)
    _lib.call("phb_advection_rhs", ct.byref(domain.desc()), domain._u_block.data_ptr(), src, mode,
              domain.velocityRHS.data_ptr(), _S(domain))
    if flags & NON_ORTHO_RHS:
        _lib.call("phb_nonortho_rhs", ct.byref(_desc(domain, flags)), _lib.PHB_NONORTHO_VELOCITY,
                  domain.velocityResult.data_ptr(), None, None, domain.velocityRHS.data_ptr(), _S(domain))


def SetupAdvectionScalar(domain: Domain, timeStep, nonOrthoFlags=0) -> None:
    """Passive-scalar right-hand side into ``domain.scalarRHS`` [B][channels][cells]
    (advection.cu:545-698, bindings SetupAdvectionScalar)."""
    _check(domain)
    flags = _flags(nonOrthoFlags)
    domain.setTimeStep(timeStep)
    sc = domain._scalar_struct()
    _lib.call("phb_scalar_rhs", ct.byref(domain.desc()), domain._phi_block.data_ptr(), domain._u_block.data_ptr(),
              ct.byref(sc), domain.scalarRHS.data_ptr(), _S(domain))
    if flags & NON_ORTHO_RHS:
        # the cross terms of scalarResult (CopyScalarResultFromBlocks before the first pass)
        _lib.call("phb_nonortho_rhs", ct.byref(_desc(domain, flags)), _lib.PHB_NONORTHO_SCALAR,
                  domain.scalarResult.data_ptr(), ct.byref(sc), None, domain.scalarRHS.data_ptr(), _S(domain))


# --- pressure ---------------------------------------------------------------------------
def SetupPressureMatrix(domain: Domain, timeStep, nonOrthoMode=0, useFaceTransform: bool = False) -> None:
    """Pressure Laplacian P = div(A^-1 grad) (pressure.cu:26-191), with the non-orthogonal
    matrix terms of ``nonOrthoMode``."""
    _check(domain)
    desc = _desc(domain, _flags(nonOrthoMode))
    if useFaceTransform:
        raise NotImplementedError("face transforms (an experimental option of the reference) are not implemented")
    domain.setTimeStep(timeStep)
    lo = _lo(domain, "P")
    _lib.call("phb_pressure_matrix", ct.byref(desc), domain.A.data_ptr(), domain._P_st.data_ptr(),
              lo.data_ptr() if lo is not None else None, _S(domain))
    _assembled(domain, "P", lo)


def SetupPressureRHS(domain: Domain, timeStep, nonOrthoMode=0, useFaceTransform: bool = False,
                     timeStepNorm: bool = False) -> None:
    """HbyA into ``pressureRHS`` and its divergence into ``pressureRHSdiv``
    (pressure.cu:350-521, :756-801)."""
    _check(domain)
    _flags(nonOrthoMode)
    if useFaceTransform or timeStepNorm:
        raise NotImplementedError("face transforms and time step normalisation are not implemented")
    domain.setTimeStep(timeStep)
    src, mode = _src(domain)
    _lib.call("phb_pressure_rhs", ct.byref(domain.desc()), domain._C_st.data_ptr(), domain.A.data_ptr(),
              domain._u_block.data_ptr(), domain.velocityResult.data_ptr(), src, mode, domain.pressureRHS.data_ptr(),
              _S(domain))
    SetupPressureRHSdiv(domain, timeStep, nonOrthoMode, useFaceTransform, timeStepNorm)


def SetupPressureRHSdiv(domain: Domain, timeStep, nonOrthoMode=0, useFaceTransform: bool = False,
                        timeStepNorm: bool = False) -> None:
    """div(pressureRHS) into ``pressureRHSdiv`` (pressure.cu:756-801), plus the
    non-orthogonal terms of ``pressureResult`` weighted with 1/A (pressure.cu:839-860)."""
    _check(domain)
    flags = _flags(nonOrthoMode)
    if useFaceTransform or timeStepNorm:
        raise NotImplementedError("face transforms and time step normalisation are not implemented")
    _lib.call("phb_divergence", ct.byref(domain.desc()), domain.pressureRHS.data_ptr(),
              domain.pressureRHSdiv.data_ptr(), _S(domain))
    if flags & NON_ORTHO_RHS:
        _lib.call("phb_nonortho_rhs", ct.byref(_desc(domain, flags)), _lib.PHB_NONORTHO_PRESSURE,
                  domain.pressureResult.data_ptr(), None, domain.A.data_ptr(), domain.pressureRHSdiv.data_ptr(),
                  _S(domain))


def ComputeVelocityDivergence(domain: Domain) -> torch.Tensor:
    """Flux divergence of the block velocity, [B * n] (piso/analysis.cu:27-70, bound at
    bindings.cpp:664): the face fluxes of the velocity interpolated to the faces (fixed
    faces take their boundary velocity), summed per cell, as for the pressure right-hand
    side's divergence."""
    _check(domain)
    div = torch.zeros_like(domain.pressureResult)
    _lib.call("phb_divergence", ct.byref(domain.desc()), domain._u_block.data_ptr(), div.data_ptr(), _S(domain))
    return div


def SetupPressureCorrection(domain: Domain, timeStep, nonOrthoMode=0, useFaceTransform: bool = False,
                            timeStepNorm: bool = False) -> None:
    """Matrix, HbyA and divergence of one corrector (pressure.cu:882-927)."""
    SetupPressureMatrix(domain, timeStep, nonOrthoMode, useFaceTransform)
    SetupPressureRHS(domain, timeStep, nonOrthoMode, useFaceTransform, timeStepNorm)


def CorrectVelocity(domain: Domain, timeStep, version: int = 0, timeStepNorm: bool = False) -> None:
    """u = HbyA - grad(p)/A into ``velocityResult`` (velocity_correction.cu:27-60). The
    pressure is read from the blocks, as in phiPICT (CopyPressureResultToBlocks first)."""
    _check(domain)
    if version not in (0, 1):
        raise NotImplementedError("phipict_b200 implements the finite-difference corrector (version 1)")
    if timeStepNorm:
        raise NotImplementedError("time step normalisation is not implemented")
    _lib.call("phb_correct_velocity", ct.byref(domain.desc()), domain._p_block.data_ptr(),
              domain.pressureRHS.data_ptr(), domain.A.data_ptr(), domain.velocityResult.data_ptr(), _S(domain))


# --- result copies (piso/result_copy.cu): one flat device copy each ----------------------
def CopyVelocityResultToBlocks(domain: Domain) -> None:
    domain._u_block.view(-1).copy_(domain.velocityResult)


def CopyVelocityResultFromBlocks(domain: Domain) -> None:
    domain.velocityResult.copy_(domain._u_block.view(-1))


def CopyPressureResultToBlocks(domain: Domain) -> None:
    domain._p_block.view(-1).copy_(domain.pressureResult)


def CopyPressureResultFromBlocks(domain: Domain) -> None:
    domain.pressureResult.copy_(domain._p_block.view(-1))


def CopyScalarResultToBlocks(domain: Domain) -> None:
    domain._phi_block.view(-1).copy_(domain.scalarResult)


def CopyScalarResultFromBlocks(domain: Domain) -> None:
    domain.scalarResult.copy_(domain._phi_block.view(-1))


def CopyEpotResultToBlocks(domain: Domain) -> None:
    domain._epot_block.view(-1).copy_(domain.epotResult)


def CopyEpotResultFromBlocks(domain: Domain) -> None:
    domain.epotResult.copy_(domain._epot_block.view(-1))


# --- MHD --------------------------------------------------------------------------------
def SetupEpotMatrix(domain: Domain, nonOrthoFlags=0, useFaceTransform: bool = False) -> None:
    domain.SetupEpotOnDomain(nonOrthoFlags, useFaceTransform)


def ComputeEpotRHS(domain: Domain, vectorField: torch.Tensor) -> torch.Tensor:
    """div(field) with the potential boundary fluxes (mhd/potential.cu:273-366)."""
    _check(domain)
    n = domain.getTotalSize() * domain.getSpatialDims() * domain.getBatchSize()
    if vectorField.dim() != 1 or vectorField.numel() != n:
        raise RuntimeError("vectorField size must be totalSize * spatialDims (* batch size).")
    if vectorField.dtype != domain.getDtype() or vectorField.device != domain.getDevice():
        raise RuntimeError("vectorField must match the domain dtype and device")
    f = vectorField.contiguous()
    out = torch.zeros(domain.getTotalSize() * domain.getBatchSize(), dtype=domain.getDtype(), device=domain.getDevice())
    _lib.call("phb_epot_rhs", ct.byref(domain.desc()), f.data_ptr(), out.data_ptr(), _S(domain))
    return out


def ComputeCurrentDensityFaceBased(domain: Domain, epotField: torch.Tensor, uCrossBField: torch.Tensor) -> torch.Tensor:
    """Face-based current density J, flat ``[B*3*cells]`` (mhd/potential.cu:718-977)."""
    _check(domain)
    d, B, N = domain.getSpatialDims(), domain.getBatchSize(), domain.getTotalSize()
    if epotField.numel() != B * N:
        raise RuntimeError("epotField size must equal domain totalSize (* batch size).")
    if uCrossBField.numel() != B * N * 3:
        if d == 3 and uCrossBField.numel() == B * N * d:
            pass
        else:
            raise RuntimeError("uCrossBField must hold 3 components per cell")
    J = torch.zeros(B * 3 * N, dtype=domain.getDtype(), device=domain.getDevice())
    e_b = torch.zeros(B, 3, dtype=torch.float64, device=domain.getDevice())
    _lib.call("phb_current_lorentz", ct.byref(domain.desc()), epotField.contiguous().data_ptr(),
              uCrossBField.contiguous().data_ptr(), e_b.data_ptr(), None, J.data_ptr(), None, 0, _S(domain))
    return J


# --- linear solves ----------------------------------------------------------------------
def SolveLinear(A: CSRmatrix, RHS: torch.Tensor, x: torch.Tensor, maxit, tol, conv=None, useBiCG: bool = False,
                matrixRankDeficient: bool = False, residualResetSteps: int = 0, transposeA: bool = False,
                printResidual: bool = False, returnBestResult: bool = False,
                BiCGwithPreconditioner: bool = False) -> list[LinearSolverResultInfo]:
    """Solve ``A x = RHS`` in place (solvers/linear_solve.cu:22-162). ``A`` must be one of
    a domain's matrices (C, P or Epot); right-hand sides per instance = RHS size / rows.

    conv: NORM2_NORMALIZED (None: the same) or NORM2, which tests ||r||_2 < tol and is run as
    NORM2_NORMALIZED with tol / sqrt(rows per instance). matrixRankDeficient: phiPICT hands a
    singular (pure Neumann) system to its legacy CG, which adds a constant-mode term to A; here
    CG runs on the system as given, which converges on the consistent (mean-free) right-hand
    sides that phiPICT's driver passes. The ABS_* criteria, preconditioned BiCGStab and
    residual resets are refused."""
    from .solvers import ConvergenceCriterion

    src = A.stencil_source() if isinstance(A, CSRmatrix) else None
    if src is None:
        raise NotImplementedError("phipict_b200 solves the stencil matrices of a Domain (C, P, Epot)")
    crit = ConvergenceCriterion.NORM2_NORMALIZED if conv is None else ConvergenceCriterion(int(conv))
    if crit not in (ConvergenceCriterion.NORM2, ConvergenceCriterion.NORM2_NORMALIZED):
        raise NotImplementedError(f"convergence criterion {crit.name} is not implemented (NORM2, NORM2_NORMALIZED)")
    if BiCGwithPreconditioner and useBiCG:
        raise NotImplementedError("Jacobi-preconditioned BiCGStab is not implemented")
    if residualResetSteps:
        raise NotImplementedError("residual resets are not implemented")
    domain, which = src
    st = domain._stencil(which)
    if transposeA:
        # A^T as a stencil (the adjoint solves of phiPICT's LinearSolveFunction,
        # core/piso_diff.py:1154-1421)
        t = torch.empty_like(st)
        _lib.call("phb_transpose_stencil", ct.byref(domain.desc()), st.data_ptr(), t.data_ptr(), _S(domain))
        st = t
    B, N = domain.getBatchSize(), domain.getTotalSize()
    nrhs = RHS.numel() // (B * N)
    if nrhs * B * N != RHS.numel() or x.numel() != RHS.numel():
        raise RuntimeError("RHS/x size must be a multiple of the matrix rows")
    maxit = int(maxit.reshape(-1)[0]) if isinstance(maxit, torch.Tensor) else int(maxit)
    if isinstance(tol, torch.Tensor) and tol.numel() > 1 and tol.numel() != B * nrhs:
        raise RuntimeError("tolerance must have 1 or (batch * right-hand sides) entries")
    if crit == ConvergenceCriterion.NORM2:
        scale = 1.0 / math.sqrt(N)
        tol = tol * scale if isinstance(tol, torch.Tensor) else float(tol) * scale
    solver = solver_for(domain, BICGSTAB if useBiCG else CG, domain.getDtype(), nrhs, tag="SolveLinear")
    solver.solve(st, RHS.contiguous(), x, tol, maxit, return_best=returnBestResult)
    return solver.results()


def SparseOuterProduct(a: torch.Tensor, b: torch.Tensor, out_pattern: CSRmatrix) -> None:
    """out.value[k] = a[row(k)] * b[col(k)] on the nonzero pattern of out_pattern, written in
    place (solvers/linear_solve.cu:167-190, the cuSPARSE SDDMM a b^T sampled at the pattern):
    the gradient of a solve with respect to the matrix values. For a domain matrix the values
    go back into its stencil."""
    n = out_pattern.getRows()
    for name, v in (("a", a), ("b", b)):
        if not v.is_cuda:
            raise RuntimeError(f"{name} must be a CUDA tensor")
        if v.dim() != 1 or v.numel() != n:
            raise RuntimeError(f"Size of {name} must match matrix size.")
    val = out_pattern.value
    if a.dtype != val.dtype or b.dtype != val.dtype:
        raise RuntimeError("Data type of a and b must match the matrix.")
    row = out_pattern.row.long()
    col = out_pattern.index.long()
    rows = torch.repeat_interleave(torch.arange(n, device=a.device), row[1:] - row[:-1])
    out = (a[rows] * b[col]).to(val.dtype)
    if val.numel() != out.numel():
        raise RuntimeError("SparseOuterProduct writes one matrix (batch size 1)")
    out_pattern.value = out


def AMGPCGSolve(aRow: torch.Tensor, aCol: torch.Tensor, aVal: torch.Tensor, levels, coarsePinv: torch.Tensor,
                rhs: torch.Tensor, x: torch.Tensor, maxIterations: int, tolerance: float, normalized: bool = True,
                returnBestResult: bool = False, projectConstant: bool = False, preSweeps: int = 1,
                postSweeps: int = 1, omega: float = 2.0 / 3.0, tolerances=()) -> list[LinearSolverResultInfo]:
    """AMG-preconditioned CG on CSR matrices, solving in place in x (bindings.cpp:764-776,
    krylov.cu:1565-1612; the solver of krylov.cu:1400-1546): for callers that bring an algebraic
    hierarchy, like phiPICT's solvers/amg.py. `levels` holds, per level but the coarsest,
    (A row, A col, A val, inverse diagonal, R row, R col, R val, P row, P col, P val) with int32
    indices; coarsePinv is the coarsest level's dense pseudo-inverse, [nc, nc] or [B, nc, nc].
    rhs and x hold B environments of aRow.numel()-1 rows each; aVal and every level's A values
    and inverse diagonal are one matrix or one per environment. One result per environment."""
    def cuda_contig(name: str, t: torch.Tensor) -> None:
        if not t.is_cuda:
            raise RuntimeError("AMG tensors must be on the GPU")
        if not t.is_contiguous():
            raise RuntimeError(f"{name}: AMG tensors must be contiguous")

    if not (rhs.is_contiguous() and x.is_contiguous() and rhs.numel() == x.numel()):
        raise RuntimeError("rhs and x must be contiguous and of equal size")
    if rhs.dtype != aVal.dtype or x.dtype != aVal.dtype:
        raise RuntimeError("rhs, x and the matrix must have the same dtype")
    if aVal.dtype not in (torch.float32, torch.float64):
        raise RuntimeError("the system must be float32 or float64")
    n = aRow.numel() - 1
    if n <= 0 or rhs.numel() % n != 0:
        raise RuntimeError("rhs size must be a multiple of the matrix size")
    B = rhs.numel() // n
    hdt = coarsePinv.dtype
    if hdt not in (torch.float32, torch.float64):
        raise RuntimeError("AMG hierarchy dtype must be float32 or float64")

    def batched_stride(name: str, row, col, val) -> int:
        for t in (row, col, val):
            cuda_contig(name, t)
        if row.dtype != torch.int32 or col.dtype != torch.int32:
            raise RuntimeError("AMG index tensors must be int32")
        nnz = col.numel()
        if val.numel() != nnz and val.numel() != nnz * B:
            raise RuntimeError(f"{name}: values must hold one matrix or one per right-hand side.")
        return 0 if val.numel() == nnz else nnz

    for t in (rhs, x):
        cuda_contig("rhs/x", t)
    stride = batched_stride("system matrix", aRow, aCol, aVal)
    if len(levels) < 1:
        raise RuntimeError("AMG hierarchy needs at least one level above the coarsest")
    lv = (_lib.PhbCsrLevel * len(levels))()
    keep = []
    for i, t in enumerate(levels):
        if len(t) != 10:
            raise RuntimeError("each AMG level needs (A row, col, val, dinv, R row, col, val, P row, col, val)")
        t = [v.contiguous() for v in t]
        keep.append(t)
        if any(t[k].dtype != hdt for k in (2, 3, 6, 9)):
            raise RuntimeError("all hierarchy values must have the dtype of the coarse pseudo-inverse")
        s = batched_stride("level operator", t[0], t[1], t[2])
        nl = t[0].numel() - 1
        cuda_contig("inverse diagonal", t[3])
        if t[3].numel() != (nl * B if s else nl):
            raise RuntimeError("inverse diagonal must match the level operator(s)")
        for name, (r, c, v) in (("R", t[4:7]), ("P", t[7:10])):
            for u in (r, c, v):
                cuda_contig(name, u)
            if r.dtype != torch.int32 or c.dtype != torch.int32:
                raise RuntimeError("AMG index tensors must be int32")
            if v.numel() != c.numel():
                raise RuntimeError(f"{name}: values and column indices differ in size")
        lv[i] = _lib.PhbCsrLevel(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), s, t[3].data_ptr(),
                                 t[4].data_ptr(), t[5].data_ptr(), t[6].data_ptr(), t[7].data_ptr(), t[8].data_ptr(),
                                 t[9].data_ptr(), nl, 0)
    for i in range(len(levels)):  # R_l maps level l to the next one, P_l back
        nnext = keep[i + 1][0].numel() - 1 if i + 1 < len(levels) else coarsePinv.shape[-1]
        if keep[i][4].numel() - 1 != nnext or keep[i][7].numel() - 1 != keep[i][0].numel() - 1:
            raise RuntimeError("restriction / prolongation sizes do not chain the levels")
    if keep[0][0].numel() - 1 != n:
        raise RuntimeError("finest AMG level does not match the system matrix")
    nc = int(coarsePinv.shape[-1])
    batched = coarsePinv.dim() == 3 and B > 1
    pinv = coarsePinv.contiguous()
    cuda_contig("coarse pseudo-inverse", pinv)
    if pinv.numel() != (nc * nc * B if batched else nc * nc):
        raise RuntimeError("coarse pseudo-inverse has the wrong size")
    tols = [float(v) for v in tolerances]
    if tols and len(tols) != B:
        raise RuntimeError("tolerances must hold one value per right-hand side")
    htol = (ct.c_double * B)(*tols) if tols else None
    dt = {torch.float32: 0, torch.float64: 1}
    a = _lib.PhbCsrPcg()
    a.dtype, a.hdtype, a.n, a.nenv, a.nlevels, a.coarse_n = dt[aVal.dtype], dt[hdt], n, B, len(levels), nc
    a.coarse_batched = int(batched)
    a.maxit, a.normalized, a.return_best = int(maxIterations), int(bool(normalized)), int(bool(returnBestResult))
    a.project_constant, a.pre_sweeps, a.post_sweeps = int(bool(projectConstant)), int(preSweeps), int(postSweeps)
    a.tol, a.omega = float(tolerance), float(omega)
    a.tolerances = ct.cast(htol, ct.c_void_p) if htol is not None else None
    a.row, a.col, a.val, a.val_stride = aRow.data_ptr(), aCol.data_ptr(), aVal.data_ptr(), stride
    a.levels = ct.cast(lv, ct.c_void_p)
    a.coarse_pinv, a.b, a.x = pinv.data_ptr(), rhs.data_ptr(), x.data_ptr()
    nbytes = _lib.load().phb_csr_pcg_work_bytes(ct.byref(a))
    if nbytes < 0:
        raise RuntimeError(_lib.load().phb_last_error().decode(errors="replace"))
    work = torch.empty(max(256, int(nbytes)), dtype=torch.uint8, device=rhs.device)
    a.work = work.data_ptr()
    out = (_lib.PhbSolveResult * B)()
    with torch.cuda.device(rhs.device):
        _lib.call("phb_csr_pcg_solve", ct.byref(a), out, _lib.stream_ptr(rhs.device))
    return [LinearSolverResultInfo(o.final_residual, o.used_iterations, bool(o.converged), bool(o.finite), o.status,
                                   o.inner_iterations) for o in out]


def GetKrylovSettings() -> dict:
    from .solvers import SETTINGS

    return {"enabled": True, "useGraphs": SETTINGS["use_graphs"], "checkInterval": SETTINGS["check_interval"]}


def SetKrylovSettings(enabled: bool = True, checkInterval: int = 8, useGraphs: bool = True,
                      cgPreconditioner=None, bicgPreconditioner=None) -> None:
    """Solver launch settings (bindings.cpp:739-751). Only the fused solvers exist here, so
    ``enabled`` must stay True; preconditioners other than none are not implemented."""
    from .solvers import SETTINGS

    if not enabled:
        raise NotImplementedError("phipict_b200 has no legacy (cuBLAS/cuSPARSE) solvers")
    SETTINGS["use_graphs"] = bool(useGraphs)
    if not useGraphs:
        SETTINGS["mode"] = "host"
    elif SETTINGS["mode"] == "host":
        SETTINGS["mode"] = "persistent"
    SETTINGS["check_interval"] = max(1, int(checkInterval))


def ReleaseKrylovWorkspaces() -> None:
    _lib.call("phb_release_graphs")
