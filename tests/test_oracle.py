"""CPU oracle pinned against the reference's known answers (no GPU needed).

- constant Dirichlet potential: E phi == rhs exactly and J == 0 (tests/test_potential_bc.py:455-471)
- Dirichlet values act linearly and only at their own face cells (test_potential_bc.py:474-514)
- the analytic Hartmann profile u(y) = G/N (1 - cosh(Ha y)/cosh(Ha)) at steady state
  (examples/hartmann.py:3-5,57-86)
- solver stop rule and solutions against SciPy (tests/test_krylov.py:89-148)
- grid metrics of rectilinear cells (grid/grid_gen.cu:299-354)
"""
import math

import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

import phipict_b200 as pb
from cases import duct_3d, hartmann_2d, rotated_pair_2d, seeded_state
from oracle.oracle import OracleDomain, OracleSim


def test_rectilinear_metrics():
    dom = hartmann_2d(6, 5, device="cpu")
    od = OracleDomain(dom)
    v = dom.getBlocks()[0].vertexCoordinates[0].numpy()
    dx = np.diff(v[0][0])
    dy = np.diff(v[1][:, 0])
    T = od.Tc.reshape(5, 6, 9)
    assert np.allclose(T[..., 0], dx[None, :])          # M[0][0]
    assert np.allclose(T[..., 3], dy[:, None])          # M[1][1]
    assert np.allclose(T[..., 1], 0) and np.allclose(T[..., 2], 0)
    assert np.allclose(T[..., 8], dx[None, :] * dy[:, None])  # det = cell area
    assert np.allclose(T[..., 4], 1 / dx[None, :])      # Minv[0][0]


def test_constant_dirichlet_potential_known_answer():
    c = 0.7
    dom = duct_3d(6, 5, 4, 1, device="cpu")
    bnd = dom.getBlocks()[0].getBoundary("-y")
    bnd.setPotentialBC(pb.PotentialBC.DIRICHLET)
    bnd.setPotentialValues(torch.full((1, 1, 4, 1, 6), c, dtype=torch.float64))
    od = OracleDomain(dom)
    E, Ecol = od.laplace_matrix(epot=True)
    n = od.n
    phi = np.full(n, c)
    rhs = od.epot_rhs(np.zeros(3 * n))
    assert np.abs(od.spmv(E, phi, col=Ecol) - rhs).max() < 1e-12
    assert np.abs(rhs).max() > 0
    J = od.current_density(phi, np.zeros(3 * n))
    assert np.abs(J).max() < 1e-12


def test_dirichlet_values_linear_and_local():
    g = torch.Generator().manual_seed(5)
    vals = torch.randn(1, 1, 4, 1, 6, generator=g, dtype=torch.float64)
    mask = torch.zeros(1, 1, 4, 1, 6, dtype=torch.int8)
    mask[..., ::2] = int(pb.PotentialBC.DIRICHLET)

    def make(values):
        dom = duct_3d(6, 5, 4, 1, device="cpu")
        bnd = dom.getBlocks()[0].getBoundary("-y")
        bnd.setPotentialTypes(mask)
        if values is not None:
            bnd.setPotentialValues(values)
        return OracleDomain(dom)

    n = make(None).n
    field = torch.randn(3 * n, generator=g, dtype=torch.float64).numpy()
    phi = torch.randn(n, generator=g, dtype=torch.float64).numpy()
    ops = {}
    for key, v in (("ref", None), ("new", vals), ("dbl", 2 * vals)):
        od = make(v)
        ops[key] = (od.laplace_matrix(epot=True)[0], od.epot_rhs(field), od.current_density(phi, field))
    assert np.array_equal(ops["ref"][0], ops["new"][0]), "values must not touch the matrix"
    changed = ops["new"][1] != ops["ref"][1]
    # only cells at y == 0 under a Dirichlet mask entry change
    z, y, x = np.unravel_index(np.arange(n), (4, 5, 6))
    expect = (y == 0) & (mask[0, 0, :, 0, :].numpy()[z, x] == 2)
    assert np.array_equal(changed, expect)
    np.testing.assert_allclose(ops["dbl"][1] - ops["ref"][1], 2 * (ops["new"][1] - ops["ref"][1]), rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("bicg", [False, True])
def test_oracle_solvers_match_scipy(bicg):
    dom = hartmann_2d(10, 8, device="cpu")
    seeded_state(dom, 3)
    od = OracleDomain(dom)
    u = dom.getBlocks()[0].velocity.reshape(-1).numpy()
    Cval, A = od.advection_matrix(u, 0.01, 0.01)
    rhs = od.advection_rhs(u, None, 0.01, 0.01)[: od.n].copy()
    x = np.zeros(od.n)
    tol = 1e-12
    st, it, crit = od.solve(Cval, rhs, x, tol, 1000, bicg=bicg)
    assert st == 1 and crit < tol
    C = od.csr_matrix(Cval)
    r = rhs - C @ x
    assert np.linalg.norm(r) / math.sqrt(od.n) < 2 * tol
    assert np.allclose(x, spla.spsolve(C, rhs), rtol=1e-9)


def test_csr_pattern_rows():
    """Row sizes: 2d+1 minus prescribed faces; periodic and connected faces keep their entry."""
    od = OracleDomain(rotated_pair_2d(4, device="cpu"))
    sizes = np.diff(od.row)
    assert sizes.min() >= 3 and sizes.max() == 5
    od3 = OracleDomain(duct_3d(4, 4, 4, 2, device="cpu"))
    sizes = np.diff(od3.row)
    assert sizes.max() == 7 and sizes.min() == 4  # a corner cell of the duct keeps 3 neighbours


def test_hartmann_profile():
    """Steady Hartmann flow reproduces the analytic profile (examples/hartmann.py)."""
    Ha, Re = 10.0, 2.0
    N = Ha * Ha / Re
    G = N  # centre-line velocity ~1
    nx, ny = 4, 48
    dom = hartmann_2d(nx, ny, device="cpu", nu=1.0 / Re, grading=2.0, length=1.0)
    od = OracleDomain(dom)
    sim = OracleSim(od, np.zeros(2 * od.n), 5e-3, 1.0 / Re,
                    advection_tol=pb.SolverTolerance(rtol=1e-10), pressure_tol=pb.SolverTolerance(rtol=1e-10, atol=1e-14),
                    mhd=dict(stuart=N, e_b=[0.0, 1.0, 0.0], singular=True,
                             potential_tol=pb.SolverTolerance(rtol=1e-10, atol=1e-14)))
    base = np.zeros(2 * od.n)
    base[: od.n] = G
    for _ in range(400):
        # the example's PRE_VELOCITY_SETUP hook resets the source before the Lorentz force is added
        sim.src = base.copy()
        sim.step()
    y = dom.getBlocks()[0].getCellCoordinates()[0, 1, :, 0].numpy()
    u = sim.u[: od.n].reshape(ny, nx).mean(1)
    exact = G / N * (1 - np.cosh(Ha * y) / math.cosh(Ha))
    err = np.abs(u - exact).max() / np.abs(exact).max()
    assert err < 5e-3, err


def test_scalar_constant_field_is_steady_under_uniform_flow():
    """Passive scalar (advection.cu:27-305 forPassiveScalar, :545-698): in a fully periodic
    box a uniform, divergence-free velocity leaves a constant scalar constant, so the scalar
    matrix applied to it reproduces its right-hand side."""
    from phipict_b200.grid import rectilinear_vertices

    dom = pb.Domain(2, torch.tensor([0.05]), name="box", device="cpu", dtype=torch.float64)
    b = dom.CreateBlock(vertexCoordinates=rectilinear_vertices(np.linspace(0, 1, 9), np.linspace(0, 2, 7),
                                                               dtype=torch.float64), name="box")
    b.MakePeriodic("x")
    b.MakePeriodic("y")
    v = torch.zeros(b.velocity.shape, dtype=torch.float64)
    v[:, 0], v[:, 1] = 1.0, 0.5
    b.velocity.copy_(v)
    od = OracleDomain(dom)
    u = v.reshape(-1).numpy()
    val, _ = od.scalar_matrix(u, 0.01, 0.02, 0)
    rhs = od.scalar_rhs(np.full(od.n, 2.5), 0.01, 0.02, 0)
    assert np.abs(od.spmv(val, np.full(od.n, 2.5)) - rhs).max() < 1e-10 * np.abs(rhs).max()


def test_scalar_dirichlet_wall_value_enters_linearly():
    """A Dirichlet face value enters the scalar right-hand side linearly and only at the cells
    of that face."""
    dom = hartmann_2d(6, 5, device="cpu")
    wall = dom.getBlocks()[0].getBoundary("-y")
    od0 = OracleDomain(dom)
    phi = np.zeros(od0.n)
    r0 = od0.scalar_rhs(phi, 0.01, 0.02, 0)
    wall.setPassiveScalar(torch.full((1, 1), 3.0, dtype=torch.float64))
    r1 = OracleDomain(dom).scalar_rhs(phi, 0.01, 0.02, 0)
    changed = np.flatnonzero(np.abs(r1 - r0) > 0)
    assert changed.size == 6 and np.all(changed < 6)  # the first row of cells (y = 0)
    wall.setPassiveScalar(torch.full((1, 1), 6.0, dtype=torch.float64))
    r2 = OracleDomain(dom).scalar_rhs(phi, 0.01, 0.02, 0)
    assert np.allclose(r2 - r0, 2 * (r1 - r0), rtol=1e-12, atol=0)
