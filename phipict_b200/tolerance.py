"""Solver tolerances relative to the right-hand side (phiPICT solvers/tolerance.py).

A :class:`SolverTolerance` resolves to the absolute tolerance of the stop test
``||r||_2/sqrt(n) < tol`` as ``max(rtol*||b||_2/sqrt(n), atol, 8*eps*||b||_2/sqrt(n))``
per batched environment (tolerance.py:142-257). phipict_b200 resolves it on the device,
inside the solver's first kernel, so no solve needs a host round trip for its tolerance.
"""
from __future__ import annotations

import math
import numbers
from dataclasses import dataclass

import torch

from . import _lib

PRECISION_FLOOR_FACTOR = 8.0
ADJOINT_RTOL_FALLBACK = 1e-4
_ADJOINT_RTOL: float | None = None


def default_tolerance(dtype: torch.dtype) -> float:
    """The dtype default of piso_diff._get_solver_tolerance (core/piso_diff.py:397-421)."""
    return 1e-8 if dtype == torch.float64 else 1e-5


@dataclass(frozen=True)
class SolverTolerance:
    rtol: float | None = None
    atol: float | None = None

    def __post_init__(self) -> None:
        if self.rtol is None and self.atol is None:
            raise ValueError("SolverTolerance needs at least one of rtol, atol.")
        for name in ("rtol", "atol"):
            value = getattr(self, name)
            if value is None:
                continue
            if not isinstance(value, numbers.Real):
                raise TypeError(f"SolverTolerance.{name} must be a float or None.")
            if not float(value) > 0:
                raise ValueError(f"SolverTolerance.{name} must be positive.")

    def resolve_scale(self, scale: float, dtype: torch.dtype) -> float:
        tol = 0.0
        if self.rtol is not None:
            tol = self.rtol * scale
        if self.atol is not None:
            tol = max(tol, self.atol)
        tol = max(tol, PRECISION_FLOOR_FACTOR * torch.finfo(dtype).eps * scale)
        if not tol > 0.0:
            tol = default_tolerance(dtype)
        return float(tol)

    def resolve(self, rhs: torch.Tensor) -> float:
        n = rhs.numel()
        scale = float(torch.linalg.vector_norm(rhs.detach().to(torch.float64))) / math.sqrt(n) if n else 0.0
        return self.resolve_scale(scale, rhs.dtype)

    def resolve_batched(self, rhs: torch.Tensor, batch_size: int) -> list[float]:
        slices = rhs.detach().reshape(batch_size, -1)
        n = slices.shape[1]
        norms = torch.linalg.vector_norm(slices.to(torch.float64), dim=1)
        scales = (norms / math.sqrt(n)).tolist() if n > 0 else [0.0] * batch_size
        return [self.resolve_scale(s, rhs.dtype) for s in scales]

    def __str__(self) -> str:
        parts = []
        if self.rtol is not None:
            parts.append(f"rtol={self.rtol:g}")
        if self.atol is not None:
            parts.append(f"atol={self.atol:g}")
        return "SolverTolerance(" + ", ".join(parts) + ")"


def parse_tolerance(tol) -> float | SolverTolerance | None:
    if tol is None or isinstance(tol, SolverTolerance):
        return tol
    if isinstance(tol, torch.Tensor):
        return tol
    if not isinstance(tol, numbers.Real) or not tol > 0:
        raise ValueError("tolerance must be a positive float, SolverTolerance or None")
    return float(tol)


def set_adjoint_rtol(rtol: float | None) -> None:
    global _ADJOINT_RTOL
    if rtol is not None and not float(rtol) > 0:
        raise ValueError(f"adjoint rtol must be positive, got {rtol}.")
    _ADJOINT_RTOL = None if rtol is None else float(rtol)


def get_adjoint_rtol() -> float | None:
    return _ADJOINT_RTOL


def to_device_tolerance(tol, dtype: torch.dtype, nsys: int, device: torch.device) -> tuple[_lib.PhbTolerance, torch.Tensor | None]:
    """Encode a tolerance as the C ABI's phb_tolerance (plus a keep-alive tensor)."""
    t = _lib.PhbTolerance()
    t.floor_eps = PRECISION_FLOOR_FACTOR * torch.finfo(dtype).eps
    t.fallback = default_tolerance(dtype)
    keep = None
    if tol is None:
        t.mode = 0
        t.atol = default_tolerance(dtype)
    elif isinstance(tol, SolverTolerance):
        t.mode = 1
        t.rtol = float(tol.rtol) if tol.rtol is not None else -1.0
        t.atol = float(tol.atol) if tol.atol is not None else -1.0
    elif isinstance(tol, torch.Tensor):
        vals = tol.detach().reshape(-1).to(torch.float64)
        if vals.numel() == 1:
            t.mode = 0
            t.atol = float(vals[0])
        else:
            if vals.numel() != nsys:
                raise RuntimeError(f"tolerance has {vals.numel()} entries, expected 1 or {nsys}")
            keep = vals.to(device)
            t.mode = 2
            t.values = keep.data_ptr()
    else:
        t.mode = 0
        t.atol = float(tol)
    return t, keep
