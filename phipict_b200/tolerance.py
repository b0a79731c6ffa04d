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

    _resolve_scale = resolve_scale  # the reference's name (tolerance.py:243)

    def resolve(self, rhs: torch.Tensor) -> float:
        return self.resolve_scale(rhs_scale(rhs), rhs.dtype)

    def resolve_batched(self, rhs: torch.Tensor, batch_size: int) -> list[float]:
        slices = rhs.detach().reshape(batch_size, -1)
        n = slices.shape[1]
        norms = torch.linalg.vector_norm(slices.to(torch.float64), dim=1)
        scales = (norms / math.sqrt(n)).tolist() if n > 0 else [0.0] * batch_size
        return [self.resolve_scale(s, rhs.dtype) for s in scales]

    def __str__(self) -> str:
        parts = []
        if self.rtol is not None:
            parts.append(f"rtol={self.rtol:.03e}")
        if self.atol is not None:
            parts.append(f"atol={self.atol:.03e}")
        return "SolverTolerance(" + ", ".join(parts) + ")"


def rhs_scale(rhs: torch.Tensor) -> float:
    """||b||_2 / sqrt(n) accumulated in float64, 0.0 for an empty RHS (tolerance.py:116-139)."""
    n = rhs.numel()
    if n == 0:
        return 0.0
    return float(torch.linalg.vector_norm(rhs.detach().to(torch.float64))) / math.sqrt(n)


def parse_tolerance(spec) -> float | SolverTolerance | None:
    """Coerce a config value into a tolerance (tolerance.py:268-323): None and
    SolverTolerance pass through, real numbers (not bools) become floats, a mapping with
    `rtol`/`atol` keys becomes a SolverTolerance; other keys raise ValueError, anything
    else TypeError."""
    if spec is None or isinstance(spec, SolverTolerance):
        return spec
    if isinstance(spec, numbers.Real) and not isinstance(spec, bool):
        return float(spec)
    if hasattr(spec, "keys"):
        unknown = set(spec.keys()) - {"rtol", "atol"}
        if unknown:
            raise ValueError(f"Unknown tolerance keys {sorted(unknown)}, expected 'rtol' and/or 'atol'.")
        rtol, atol = spec.get("rtol", None), spec.get("atol", None)
        return SolverTolerance(rtol=None if rtol is None else float(rtol), atol=None if atol is None else float(atol))
    raise TypeError(f"Cannot interpret {spec!r} as a solver tolerance; expected None, a float, "
                    "a SolverTolerance, or a mapping with rtol/atol.")


def resolve_tolerance(tol, rhs: torch.Tensor, batch_size: int = 1):
    """A SolverTolerance resolved against `rhs` (a list per environment when batch_size > 1);
    any other value unchanged (tolerance.py:326-354). The solvers here resolve on the device
    instead; this host form serves callers of the reference's function."""
    if isinstance(tol, SolverTolerance):
        if batch_size > 1:
            return tol.resolve_batched(rhs, batch_size)
        return tol.resolve(rhs)
    return tol


def coerce_tolerance(tol):
    """The tolerance keyword of a simulation: what parse_tolerance accepts, or a tensor of
    per-system absolute tolerances (which the reference's solvers take unchanged)."""
    if isinstance(tol, torch.Tensor):
        return tol
    return parse_tolerance(tol)


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
