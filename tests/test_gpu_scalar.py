"""Passive-scalar transport (phiPICT's forPassiveScalar matrix, kPISO_build_scalar_advection_RHS
and the scalar stage of the PISO step) against the CPU oracle on the same seeded inputs:
Dirichlet and Neumann faces, static and varying face values, one diffusivity for all channels
or one per channel, and a default domain whose zero scalar must not change the flow."""
import numpy as np
import pytest
import torch

import phipict_b200 as pb
from phipict_b200 import _C
from phipict_b200.domain import BoundaryConditionType as BC
from cases import duct_3d, hartmann_2d, seeded_state
from oracle.oracle import OracleDomain, OracleSim

pytestmark = pytest.mark.gpu


def host(t):
    return t.detach().cpu().numpy()


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _channel_case(dtype, per_channel_nu=True):
    """2D channel, two channels: a Dirichlet wall at -y (static values), a Neumann wall at +y
    (given gradients), seeded scalar field."""
    dom = hartmann_2d(16, 12, dtype=dtype, channels=2)
    if per_channel_nu:
        dom.setPassiveScalarViscosity(torch.tensor([0.02, 0.005]))
    b = dom.getBlocks()[0]
    b.CloseBoundary("-y", passiveScalar=torch.tensor([[1.0, 0.5]], dtype=dtype, device="cuda"))
    b.CloseBoundary("+y", passiveScalar=torch.tensor([[0.3, -0.1]], dtype=dtype, device="cuda"))
    b.getBoundary("+y").setPassiveScalarType(BC.NEUMANN)
    seeded_state(dom, 3)
    g = torch.Generator().manual_seed(5)
    b.setPassiveScalar(torch.rand(b.passiveScalar.shape, generator=g, dtype=dtype).to("cuda"))
    return dom


def _duct_case(dtype):
    """3D connected duct, one channel: a varying inflow scalar, a Neumann scalar (zero
    gradient) on the flux-balanced outflow, zero walls."""
    dom = duct_3d(8, 6, 5, 2, dtype=dtype)
    seeded_state(dom, 4)
    blocks = dom.getBlocks()
    inflow = blocks[0].getBoundary("-x")
    g = torch.Generator().manual_seed(8)
    shape = [1, 1] + inflow.face_shape()
    inflow.setPassiveScalar(torch.rand(shape, generator=g, dtype=dtype).to("cuda"))
    blocks[-1].getBoundary("+x").setPassiveScalarType(BC.NEUMANN)
    for b in blocks:
        b.setPassiveScalar(torch.rand(b.passiveScalar.shape, generator=g, dtype=dtype).to("cuda"))
    return dom


CASES = {"channel2d": _channel_case, "duct3d": _duct_case}


@pytest.mark.parametrize("case", list(CASES))
def test_scalar_matrix_and_rhs_match_the_oracle(cuda, case):
    dom = CASES[case](torch.float64)
    dom.PrepareSolve()
    od = OracleDomain(dom, 0, np.float64)
    dt = 0.01
    ts = torch.tensor([dt], dtype=torch.float64)
    u = host(dom._u_block).reshape(-1)
    C = dom.getPassiveScalarChannels()
    nus = dom.passiveScalarViscosity
    _C.SetupAdvectionScalar(dom, ts, 0)
    rhs = host(dom.scalarRHS).reshape(C, -1)
    phi = host(dom._phi_block).reshape(C, -1)
    for c in range(C):
        nu = float(dom.viscosity[0]) if nus is None else float(nus[0] if nus.numel() == 1 else nus[c])
        _C.SetupAdvectionMatrix(dom, ts, 0, forPassiveScalar=True, passiveScalarChannel=c)
        val, A = od.scalar_matrix(u, dt, nu, c)
        assert rel(host(dom.C.value), val) < 1e-12
        assert rel(host(dom.A), A) < 1e-12
        assert rel(rhs[c], od.scalar_rhs(phi[c], dt, nu, c)) < 1e-12


@pytest.mark.parametrize("case", list(CASES))
def test_scalar_steps_match_the_oracle(cuda, case):
    dom = CASES[case](torch.float64)
    dom.PrepareSolve()
    od = OracleDomain(dom, 0, np.float64)
    tol = pb.SolverTolerance(rtol=1e-12, atol=1e-14)
    nus = dom.passiveScalarViscosity
    ref = OracleSim(od, host(dom._u_block).reshape(-1), 0.01, float(dom.viscosity[0]), advection_tol=tol,
                    pressure_tol=tol, scalar=dict(phi=host(dom._phi_block).reshape(-1),
                                                  nu=None if nus is None else nus.tolist()))
    sim = pb.Simulation(dom, 0.01, non_orthogonal=False, advection_tol=tol, pressure_tol=tol)
    for _ in range(3):
        assert sim.single_step(), sim.last_error
        ref.step()
    torch.cuda.synchronize()
    assert rel(host(dom._phi_block).reshape(-1), ref.phi_s.reshape(-1)) < 1e-9
    assert rel(host(dom._u_block).reshape(-1), ref.u) < 1e-9
    tags = [t for t, _ in sim.solve_report()]
    assert any(t.startswith("scalar") for t in tags)


def test_zero_scalar_of_a_default_domain_leaves_the_flow_unchanged(cuda):
    """phiPICT domains carry one scalar channel by default; transporting its zeros reuses the
    scalar matrix for the velocity (same diffusivity and face types) and gives the same bits
    as a domain without scalars."""
    out = []
    for channels in (1, 0):
        dom = duct_3d(8, 6, 5, 2, channels=channels)
        seeded_state(dom, 2)
        dom.PrepareSolve()
        tol = pb.SolverTolerance(rtol=1e-10)
        sim = pb.MHDSimulation(dom, 0.01, torch.tensor(1.0), torch.tensor([0.0, 1.0, 0.0], dtype=torch.float64),
                               non_orthogonal=False, advection_tol=tol, pressure_tol=tol, potential_tol=tol)
        for _ in range(2):
            assert sim.single_step(), sim.last_error
        torch.cuda.synchronize()
        out.append((host(dom._u_block).copy(), host(dom._p_block).copy(), dom.hasPassiveScalar()))
    assert out[0][2] and not out[1][2]
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_diffusion_between_dirichlet_walls_reaches_the_linear_profile(cuda):
    """No flow, phi = 0 at y = -1 and 1 at y = +1, periodic in x: the ghost-cell scheme is
    exact for linear fields, so the steady state is phi = (y + 1) / 2 at the cell centres."""
    from phipict_b200.grid import rectilinear_vertices

    ny = 16
    dom = pb.Domain(2, torch.tensor([0.1]), name="slab", device="cuda", dtype=torch.float64)
    b = dom.CreateBlock(vertexCoordinates=rectilinear_vertices(np.linspace(0, 1, 5), np.linspace(-1, 1, ny + 1),
                                                               dtype=torch.float64), name="slab")
    b.MakePeriodic("x")
    b.CloseBoundary("-y", passiveScalar=torch.zeros(1, 1, dtype=torch.float64, device="cuda"))
    b.CloseBoundary("+y", passiveScalar=torch.ones(1, 1, dtype=torch.float64, device="cuda"))
    dom.PrepareSolve()
    tol = pb.SolverTolerance(rtol=1e-13, atol=1e-15)
    sim = pb.Simulation(dom, 10.0, non_orthogonal=False, advection_tol=tol, pressure_tol=tol)
    for _ in range(60):
        assert sim.single_step(), sim.last_error
    torch.cuda.synchronize()
    yc = (np.arange(ny) + 0.5) / ny * 2 - 1
    want = np.broadcast_to(((yc + 1) / 2)[:, None], (ny, 4))
    assert np.abs(host(b.passiveScalar)[0, 0] - want).max() < 1e-8
