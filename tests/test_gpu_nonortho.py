"""Curvilinear (non-orthogonal) grids: the cross terms of the momentum, scalar and pressure
matrices (advection.cu:176-240, pressure.cu:103-156, nonortho_laplace.cuh:52-129), the
explicit terms of the right-hand sides (nonortho_rhs.cuh:27-180, advection.cu:684-689,
936-937, pressure.cu:839-860) with the corner values of block_data.cuh:501-620, and the step
that re-solves with them (core/piso_simulation.py:3225-3345,3839-3891,3978-4117), checked
against the CPU oracle on the same seeded inputs."""
import numpy as np
import pytest
import torch

import phipict_b200 as pb
from phipict_b200 import _C
from phipict_b200.domain import BoundaryConditionType as BC
from cases import hartmann_2d, seeded_state, skewed_channel_2d, skewed_duct_3d, skewed_pair_2d
from oracle.oracle import OracleDomain, OracleSim

pytestmark = pytest.mark.gpu

MODE = _C.NON_ORTHO_CENTER_MATRIX | _C.NON_ORTHO_DIRECT_MATRIX | _C.NON_ORTHO_DIAGONAL_RHS
ALL = MODE | _C.NON_ORTHO_DIRECT_RHS


def host(t):
    return t.detach().cpu().numpy()


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _channel():
    """Two scalar channels: varying Dirichlet values on the -y wall, a Neumann +y wall; the
    -y wall slides along x with a varying speed."""
    dom = skewed_channel_2d(12, 10, channels=2)
    dom.setPassiveScalarViscosity(torch.tensor([0.02, 0.005]))
    b = dom.getBlocks()[0]
    g = torch.Generator().manual_seed(11)
    lo = b.getBoundary("-y")
    wall = torch.zeros([1, 2] + lo.face_shape(), dtype=torch.float64)
    wall[0, 0] = 0.2 * torch.rand(lo.face_shape(), generator=g, dtype=torch.float64)
    lo.setVelocity(wall.to("cuda"))
    lo.setPassiveScalar(torch.rand([1, 2] + lo.face_shape(), generator=g, dtype=torch.float64).to("cuda"))
    b.getBoundary("+y").setPassiveScalarType(BC.NEUMANN)
    return dom


def _duct():
    dom = skewed_duct_3d(6, 5, 4, 2)
    inflow = dom.getBlocks()[0].getBoundary("-x")
    g = torch.Generator().manual_seed(12)
    inflow.setPassiveScalar(torch.rand([1, 1] + inflow.face_shape(), generator=g, dtype=torch.float64).to("cuda"))
    dom.getBlocks()[-1].getBoundary("+x").setPassiveScalarType(BC.NEUMANN)
    return dom


CASES = {"channel2d": _channel, "duct3d": _duct, "pair2d": lambda: skewed_pair_2d(6)}


def _setup(case, seed=0):
    dom = CASES[case]()
    seeded_state(dom, seed, scale=0.3)
    g = torch.Generator().manual_seed(seed + 20)
    for b in dom.getBlocks():
        b.setPassiveScalar(torch.rand(b.passiveScalar.shape, generator=g, dtype=torch.float64).to("cuda"))
    dom.PrepareSolve()
    return dom, OracleDomain(dom)


@pytest.mark.parametrize("flags", [MODE, ALL], ids=["mode", "all"])
@pytest.mark.parametrize("case", list(CASES))
def test_nonortho_assembly_matches_the_oracle(cuda, case, flags):
    dom, od = _setup(case)
    assert dom.hasNonOrthogonalMetrics()
    dt, nu = 0.01, float(dom.viscosity[0])
    ts = torch.tensor([dt], dtype=torch.float64)
    n, d = od.n, od.dims
    u = host(dom._u_block).reshape(-1)
    g = torch.Generator().manual_seed(3)
    # momentum matrix and right-hand side with the cross terms of a velocity result
    _C.SetupAdvectionMatrix(dom, ts, flags)
    Cval, A = od.advection_matrix(u, dt, nu, flags=flags)
    assert rel(host(dom.C.value), Cval) < 1e-12 and rel(host(dom.A), A) < 1e-12
    assert rel(Cval, od.advection_matrix(u, dt, nu)[0]) > 1e-6  # the cross terms are there
    ures = u + 0.2 * torch.randn(u.size, generator=g, dtype=torch.float64).numpy()
    dom.velocityResult.copy_(torch.from_numpy(ures).to("cuda"))
    _C.SetupAdvectionVelocity(dom, ts, flags, False)
    assert rel(host(dom.velocityRHS), od.advection_rhs(u, None, dt, nu, flags=flags, ures=ures)) < 1e-12
    # pressure matrix, HbyA and its divergence with the cross terms of a pressure result
    _C.SetupPressureMatrix(dom, ts, flags, False)
    Pval, _ = od.laplace_matrix(A, flags=flags)
    assert rel(host(dom.P.value), Pval) < 1e-12
    pres = torch.randn(n, generator=g, dtype=torch.float64).numpy()
    dom.pressureResult.copy_(torch.from_numpy(pres).to("cuda"))
    _C.SetupPressureRHS(dom, ts, flags, False, False)
    h = od.pressure_rhs(Cval, A, u, ures, None, dt, nu)
    assert rel(host(dom.pressureRHS), h) < 1e-12
    assert rel(host(dom.pressureRHSdiv), od.pressure_nonortho(A, pres, flags, od.divergence(h))) < 1e-12
    # scalar matrices and right-hand side with the cross terms of a scalar result
    C = dom.getPassiveScalarChannels()
    if C == 0:
        return
    nus = dom.passiveScalarViscosity
    nu_of = (lambda c: nu) if nus is None else (lambda c: float(nus[0] if nus.numel() == 1 else nus[c]))
    for c in range(C):
        _C.SetupAdvectionMatrix(dom, ts, flags, forPassiveScalar=True, passiveScalarChannel=c)
        assert rel(host(dom.C.value), od.scalar_matrix(u, dt, nu_of(c), c, flags=flags)[0]) < 1e-12
    phi = host(dom._phi_block).reshape(C, n)
    phires = phi + 0.3 * torch.randn(C, n, generator=g, dtype=torch.float64).numpy()
    dom.scalarResult.copy_(torch.from_numpy(phires.reshape(-1)).to("cuda"))
    _C.SetupAdvectionScalar(dom, ts, flags)
    rhs = host(dom.scalarRHS).reshape(C, n)
    for c in range(C):
        ref = od.scalar_rhs(phi[c], dt, nu_of(c), c, u=u, flags=flags, phires=phires[c])
        assert rel(rhs[c], ref) < 1e-12, c


def test_rectilinear_grids_skip_the_cross_terms(cuda):
    dom = hartmann_2d(8, 6)
    dom.PrepareSolve()
    assert not dom.hasNonOrthogonalMetrics()
    assert pb.Simulation(dom, 0.01)._nonortho_flags() == 0
    sk = skewed_channel_2d(8, 6)
    sk.PrepareSolve()
    assert pb.Simulation(sk, 0.01)._nonortho_flags() == MODE
    assert pb.Simulation(sk, 0.01, non_orthogonal=False)._nonortho_flags() == 0


@pytest.mark.parametrize("case,steps", [("channel2d", (1, 1)), ("channel2d", (2, 2)), ("duct3d", (1, 1))],
                         ids=["channel2d", "channel2d-resolve", "duct3d"])
def test_nonortho_steps_match_the_oracle(cuda, case, steps):
    """Whole steps with phiPICT's non-orthogonal mode; the non-symmetric pressure systems are
    solved with BiCGStab on both sides."""
    dom, od = _setup(case, seed=5)
    tol = pb.SolverTolerance(rtol=1e-12, atol=1e-14)
    nus = dom.passiveScalarViscosity
    ref = OracleSim(od, host(dom._u_block).reshape(-1), 0.01, float(dom.viscosity[0]), advection_tol=tol,
                    pressure_tol=tol, scalar=dict(phi=host(dom._phi_block).reshape(-1),
                                                  nu=None if nus is None else host(nus)),
                    nonortho_flags=MODE, advect_non_ortho_steps=steps[0], pressure_non_ortho_steps=steps[1],
                    pressure_bicg=True)
    sim = pb.Simulation(dom, 0.01, advection_tol=tol, pressure_tol=tol, pressure_use_BiCG=True,
                        advect_non_ortho_steps=steps[0], pressure_non_ortho_steps=steps[1])
    for _ in range(3):
        assert sim.single_step(), sim.last_error
        ref.step()
    torch.cuda.synchronize()
    assert rel(host(dom._u_block).reshape(-1), ref.u) < 1e-9
    assert rel(host(dom.pressureResult), ref.p) < 1e-8
    assert rel(host(dom._phi_block).reshape(-1), ref.phi_s.reshape(-1)) < 1e-9


def test_orthogonal_step_on_a_curvilinear_grid(cuda):
    """non_orthogonal=False ignores the cross terms, as phiPICT's orthogonal path does."""
    dom, od = _setup("channel2d", seed=6)
    tol = pb.SolverTolerance(rtol=1e-12, atol=1e-14)
    nus = dom.passiveScalarViscosity
    ref = OracleSim(od, host(dom._u_block).reshape(-1), 0.01, float(dom.viscosity[0]), advection_tol=tol,
                    pressure_tol=tol, scalar=dict(phi=host(dom._phi_block).reshape(-1), nu=host(nus)))
    sim = pb.Simulation(dom, 0.01, advection_tol=tol, pressure_tol=tol, non_orthogonal=False)
    for _ in range(2):
        assert sim.single_step(), sim.last_error
        ref.step()
    torch.cuda.synchronize()
    assert rel(host(dom._u_block).reshape(-1), ref.u) < 1e-9


def test_nonortho_mhd_steps_match_the_oracle(cuda):
    """The MHD step on the curvilinear duct: non-orthogonal momentum and pressure, the
    potential with its own flags at phiPICT's default 0."""
    dom = skewed_duct_3d(6, 5, 4, 2)
    seeded_state(dom, 9, scale=0.1)
    dom.PrepareSolve()
    od = OracleDomain(dom)
    tol = pb.SolverTolerance(rtol=1e-12, atol=1e-14)
    N, e_b = 2.0, [0.0, 1.0, 0.0]
    ref = OracleSim(od, host(dom._u_block).reshape(-1), 0.01, float(dom.viscosity[0]), advection_tol=tol,
                    pressure_tol=tol, mhd=dict(stuart=N, e_b=e_b, singular=True, potential_tol=tol),
                    scalar=dict(phi=host(dom._phi_block).reshape(-1), nu=None), nonortho_flags=MODE, pressure_bicg=True)
    sim = pb.MHDSimulation(dom, 0.01, torch.tensor(N), torch.tensor(e_b, dtype=torch.float64), advection_tol=tol,
                           pressure_tol=tol, potential_tol=tol, pressure_use_BiCG=True)
    for _ in range(3):
        assert sim.single_step(), sim.last_error
        ref.step()
    torch.cuda.synchronize()
    assert rel(host(dom._u_block).reshape(-1), ref.u) < 1e-8
    assert rel(host(dom.epotResult), ref.phi) < 1e-7


def test_nonortho_batch_equals_instances_alone(cuda):
    """Curvilinear domains of different grids and viscosities batched into one descriptor step
    exactly as they do alone."""
    def members():
        out = []
        for k, (nx, ny, nu, shear) in enumerate(((12, 10, 0.02, 0.35), (14, 8, 0.03, 0.2))):
            dom = skewed_channel_2d(nx, ny, nu=nu, shear=shear, channels=0)
            seeded_state(dom, 60 + k, scale=0.2)
            dom.PrepareSolve()
            out.append(dom)
        return out

    tol = pb.SolverTolerance(rtol=1e-12, atol=1e-14)
    kw = dict(advection_tol=tol, pressure_tol=tol, pressure_use_BiCG=True)
    alone = []
    for dom in members():
        sim = pb.Simulation(dom, 0.01, **kw)
        for _ in range(3):
            assert sim.single_step(), sim.last_error
        alone.append((dom._u_block.clone(), dom.pressureResult.clone()))
    ms = members()
    batch = pb.DomainBatch(ms)
    assert batch.hasNonOrthogonalMetrics()
    sim = pb.Simulation(batch, 0.01, **kw)
    for _ in range(3):
        assert sim.single_step(), sim.last_error
    batch.scatter()
    for k, dom in enumerate(ms):
        assert torch.equal(dom._u_block, alone[k][0]), k
        assert torch.equal(dom.pressureResult, alone[k][1]), k


def test_nonortho_assembly_float32(cuda):
    """The float32 instantiations against the oracle in float32 (FP32 bar 1e-5)."""
    dom = skewed_channel_2d(12, 10, dtype=torch.float32)
    seeded_state(dom, 2, scale=0.3)
    dom.PrepareSolve()
    od = OracleDomain(dom, 0, np.float32)
    dt, nu = 0.01, float(dom.viscosity[0])
    ts = torch.tensor([dt], dtype=torch.float64)
    u = host(dom._u_block).reshape(-1)
    _C.SetupAdvectionMatrix(dom, ts, ALL)
    Cval, A = od.advection_matrix(u, dt, nu, flags=ALL)
    assert rel(host(dom.C.value), Cval) < 1e-5 and rel(host(dom.A), A) < 1e-5
    g = torch.Generator().manual_seed(4)
    ures = (u + 0.2 * torch.randn(u.size, generator=g, dtype=torch.float64).numpy()).astype(np.float32)
    dom.velocityResult.copy_(torch.from_numpy(ures).to("cuda"))
    _C.SetupAdvectionVelocity(dom, ts, ALL, False)
    assert rel(host(dom.velocityRHS), od.advection_rhs(u, None, dt, nu, flags=ALL, ures=ures)) < 1e-5
    _C.SetupPressureMatrix(dom, ts, ALL, False)
    assert rel(host(dom.P.value), od.laplace_matrix(A, flags=ALL)[0]) < 1e-5
    pres = torch.randn(od.n, generator=g, dtype=torch.float64).numpy().astype(np.float32)
    dom.pressureResult.copy_(torch.from_numpy(pres).to("cuda"))
    _C.SetupPressureRHS(dom, ts, ALL, False, False)
    h = od.pressure_rhs(Cval, A, u, ures, None, dt, nu)
    assert rel(host(dom.pressureRHSdiv), od.pressure_nonortho(A, pres, ALL, od.divergence(h))) < 1e-5
