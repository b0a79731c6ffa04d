"""Grid construction helpers (setup only): cell weight distributions and rectilinear
vertex grids, in the layout phiPICT's ``CreateBlock(vertexCoordinates=...)`` takes,
``[1, dims, (z+1), y+1, x+1]``."""
from __future__ import annotations

import numpy as np
import torch


def make_weights_tanh(res: int, A: float, refinement: str = "BOTH") -> list[float]:
    """Classical tanh stretching (grid/shapes.py:938-994): ``res+1`` weights in [0, 1]."""
    if abs(A) < 1e-10:
        return np.linspace(0.0, 1.0, res + 1).tolist()
    if refinement == "START":
        xi = np.linspace(-1, 0, res + 1)
        w = np.tanh(A * xi) / np.tanh(A) + 1.0
    elif refinement == "END":
        xi = np.linspace(0, 1, res + 1)
        w = np.tanh(A * xi) / np.tanh(A)
    elif refinement == "BOTH":
        xi = np.linspace(-1, 1, res + 1)
        w = 0.5 * (np.tanh(A * xi) / np.tanh(A)) + 0.5
    else:
        raise ValueError(f"Unknown refinement '{refinement}'. Use 'START', 'END', or 'BOTH'.")
    w[0] = 0.0
    w[-1] = 1.0
    return w.tolist()


def make_weights_simple(res: int, grading: float, refinement: str = "BOTH") -> list[float]:
    """OpenFOAM-style simpleGrading (grid/shapes.py:795-877): cell sizes in geometric
    progression with last/first ratio ``grading``; "BOTH" grades each half towards its wall
    (the first res//2 cells growing, the rest shrinking). ``res+1`` weights in [0, 1]."""

    def sizes_of(n: int) -> np.ndarray:
        if abs(grading - 1.0) < 1e-10:
            return np.full(n, 1.0 / n)
        q = grading ** (1.0 / (n - 1))
        s = q ** np.arange(n, dtype=np.float64)
        return s / s.sum()

    if refinement == "START":
        sizes = sizes_of(res)
    elif refinement == "END":
        sizes = sizes_of(res)[::-1]
    elif refinement == "BOTH":
        half = res // 2
        sizes = np.concatenate([sizes_of(half), sizes_of(res - half)[::-1]])
    else:
        raise ValueError(f"Unknown refinement '{refinement}'. Use 'START', 'END', or 'BOTH'.")
    sizes = sizes / sizes.sum()
    return [0.0] + np.cumsum(sizes).tolist()


def make_weights(grading_type: str, res: int, grading: float, refinement: str = "BOTH") -> list[float]:
    """Cell weights of a grading scheme by name (grid/shapes.py:996-1036): "simple" or "tanh"."""
    if grading_type == "simple":
        return make_weights_simple(res, grading, refinement)
    if grading_type == "tanh":
        return make_weights_tanh(res, grading, refinement)
    raise ValueError(f"Unknown grading type '{grading_type}'. Use 'simple' or 'tanh'.")


def make_weights_uniform(res: int) -> list[float]:
    return np.linspace(0.0, 1.0, res + 1).tolist()


def rectilinear_vertices(xs, ys, zs=None, dtype: torch.dtype = torch.float64) -> torch.Tensor:
    """Tensor-product vertices from 1D coordinate lists: ``[1, 2, ny+1, nx+1]`` in 2D,
    ``[1, 3, nz+1, ny+1, nx+1]`` in 3D."""
    x = torch.as_tensor(np.asarray(xs, dtype=np.float64))
    y = torch.as_tensor(np.asarray(ys, dtype=np.float64))
    if zs is None:
        Y, X = torch.meshgrid(y, x, indexing="ij")
        return torch.stack([X, Y]).unsqueeze(0).to(dtype).contiguous()
    z = torch.as_tensor(np.asarray(zs, dtype=np.float64))
    Z, Y, X = torch.meshgrid(z, y, x, indexing="ij")
    return torch.stack([X, Y, Z]).unsqueeze(0).to(dtype).contiguous()


def span(lo: float, hi: float, weights) -> np.ndarray:
    w = np.asarray(weights, dtype=np.float64)
    return lo + (hi - lo) * w


def cell_centers(vertices: torch.Tensor) -> torch.Tensor:
    """Cell centre coordinates ``[dims, (z,) y, x]`` of a vertex tensor."""
    c = vertices[0]
    for ax in range(c.dim() - 1):
        dim = 1 + ax
        c = 0.5 * (c.narrow(dim, 0, c.shape[dim] - 1) + c.narrow(dim, 1, c.shape[dim] - 1))
    return c
