"""The oracle's non-orthogonal terms (nonortho_laplace.cuh, nonortho_rhs.cuh, the corner
values of block_data.cuh:501-620) checked on the CPU by what the discretisation must do:

- on a rectilinear grid every cross term is exactly zero, so the flags change nothing;
- on an affine (uniformly sheared) grid the full discrete Laplacian, matrix part plus the
  explicit cross terms of the same field, of a linear field vanishes at interior cells, for
  the pressure operator (weights 1/A) and the viscous operator of the momentum and scalar
  equations (weights nu); without the cross terms it does not.
"""
import numpy as np
import pytest
import torch

import phipict_b200 as pb
from phipict_b200 import _C
from phipict_b200.grid import rectilinear_vertices
from cases import duct_3d, hartmann_2d
from oracle.oracle import OracleDomain

MODE = _C.NON_ORTHO_CENTER_MATRIX | _C.NON_ORTHO_DIRECT_MATRIX | _C.NON_ORTHO_DIAGONAL_RHS
ALL = MODE | _C.NON_ORTHO_DIRECT_RHS


def _sheared_box(d, n, shear=(0.35, 0.2), nu=0.03):
    """Uniform grid of the unit box, x sheared by shear . (y, z): an affine map. Periodic
    in x, walls elsewhere."""
    xs = np.linspace(0.0, 1.0, n[0] + 1)
    ys = np.linspace(0.0, 1.0, n[1] + 1)
    zs = np.linspace(0.0, 1.0, n[2] + 1) if d == 3 else None
    v = rectilinear_vertices(xs, ys, zs)
    v[0, 0] = v[0, 0] + shear[0] * v[0, 1] + (shear[1] * v[0, 2] if d == 3 else 0)
    dom = pb.Domain(d, torch.tensor([nu]), device="cpu", dtype=torch.float64)
    b = dom.CreateBlock(vertexCoordinates=v)
    for f in ("-y", "+y") + (("-z", "+z") if d == 3 else ()):
        b.CloseBoundary(f)
    b.MakePeriodic("x")
    return dom


def _centres(od, dom):
    """Cell centres [d][n] of the single block."""
    v = dom.getBlocks()[0].vertexCoordinates[0].numpy()
    c = v
    for ax in range(1, v.ndim):
        c = 0.5 * (np.take(c, range(c.shape[ax] - 1), axis=ax) + np.take(c, range(1, c.shape[ax]), axis=ax))
    return c.reshape(od.dims, -1)


def _interior(dom, margin=2):
    """Cells at least `margin` cells away from the walls and from the periodic seam in x
    (where a linear field in x jumps)."""
    nx, ny, nz = dom.getBlocks()[0].getSizes()
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    keep = (y >= margin) & (y < ny - margin) & (x >= margin) & (x < nx - margin)
    if dom.getSpatialDims() == 3:
        keep &= (z >= margin) & (z < nz - margin)
    return keep.reshape(-1)


@pytest.mark.parametrize("make", [lambda: hartmann_2d(8, 6, device="cpu"), lambda: duct_3d(5, 4, 4, 2, device="cpu")],
                         ids=["channel2d", "duct3d"])
def test_rectilinear_grid_has_no_cross_terms(make):
    dom = make()
    od = OracleDomain(dom)
    g = np.random.default_rng(0)
    u = g.standard_normal(od.dims * od.n)
    ures = g.standard_normal(od.dims * od.n)
    p = g.standard_normal(od.n)
    for flags in (MODE, ALL):
        C0, A0 = od.advection_matrix(u, 0.01, 0.02)
        C1, A1 = od.advection_matrix(u, 0.01, 0.02, flags=flags)
        assert np.array_equal(C0, C1) and np.array_equal(A0, A1)
        P0, _ = od.laplace_matrix(A0)
        P1, _ = od.laplace_matrix(A0, flags=flags)
        assert np.array_equal(P0, P1)
        r0 = od.advection_rhs(u, None, 0.01, 0.02)
        r1 = od.advection_rhs(u, None, 0.01, 0.02, flags=flags, ures=ures)
        assert np.array_equal(r0, r1)
        div = g.standard_normal(od.n)
        assert np.array_equal(od.pressure_nonortho(A0, p, flags, div), div)


def _harmonic_fields(c):
    """Fields whose physical Laplacian is zero: linear ones and harmonic quadratics (the
    quadratics have cross derivatives, so only the non-orthogonal terms get them right)."""
    f = {"x": c[0], "y": c[1], "xy": c[0] * c[1], "x2-y2": c[0] ** 2 - c[1] ** 2}
    if c.shape[0] == 3:
        f.update({"z": c[2], "xz": c[0] * c[2], "yz": c[1] * c[2]})
    return f


@pytest.mark.parametrize("d,n", [(2, (10, 9, 1)), (3, (7, 7, 6))])
@pytest.mark.parametrize("flags", [MODE, ALL], ids=["mode", "direct_rhs"])
def test_pressure_laplacian_of_harmonic_fields_vanishes_on_an_affine_grid(d, n, flags):
    dom = _sheared_box(d, n)
    od = OracleDomain(dom)
    A = np.ones(od.n)
    keep = _interior(dom)
    P, col = od.laplace_matrix(A, flags=flags)
    P0, col0 = od.laplace_matrix(A)
    for name, p in _harmonic_fields(_centres(od, dom)).items():
        L = od.spmv(P, p, col=col) - od.pressure_nonortho(A, p, flags, np.zeros(od.n))
        assert np.abs(L[keep]).max() < 1e-13, (name, np.abs(L[keep]).max())
        if name == "xy":  # the orthogonal operator alone misses the cross derivative
            assert np.abs(od.spmv(P0, p, col=col0)[keep]).max() > 1e-4


@pytest.mark.parametrize("d,n", [(2, (10, 9, 1)), (3, (7, 7, 6))])
@pytest.mark.parametrize("flags", [MODE, ALL], ids=["mode", "direct_rhs"])
def test_viscous_laplacian_of_harmonic_fields_vanishes_on_an_affine_grid(d, n, flags):
    """det C x - det x / dt + S(x) (S: the explicit cross terms the momentum right-hand side
    subtracts) is the discrete -nu Laplacian of x when the flow is at rest."""
    dom = _sheared_box(d, n)
    od = OracleDomain(dom)
    dt, nu = 0.5, 0.03
    u0 = np.zeros(d * od.n)
    C, A = od.advection_matrix(u0, dt, nu, flags=flags)
    det = od.Tc[:, -1]
    keep = _interior(dom)
    r0 = od.advection_rhs(u0, None, dt, nu)
    for name, f in _harmonic_fields(_centres(od, dom)).items():
        x = np.zeros(d * od.n)
        x[:od.n] = f
        S = (r0 - od.advection_rhs(u0, None, dt, nu, flags=flags, ures=x))[:od.n] * det
        L = det * od.spmv(C, f) - det * f / dt + S
        assert np.abs(L[keep]).max() < 1e-13, (name, np.abs(L[keep]).max())
