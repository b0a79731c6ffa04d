"""LINEAR_UPWIND advection (domain_structs_gpu.h:65-68): first-order upwind in the momentum and
scalar matrices where the far-upwind cell lies in the block (shared_stencils.cuh:35-43), with
the linear-upwind part as a lagged explicit correction in the momentum right-hand side
(advection.cu:892-934), repeated in HbyA (pressure.cu:474-515), and in the scalar right-hand
side (advection.cu:652-688); checked against the CPU oracle on the same seeded inputs."""
import numpy as np
import pytest
import torch

import phipict_b200 as pb
from phipict_b200 import _C
from phipict_b200.domain import AdvectionScheme
from cases import duct_3d, hartmann_2d, seeded_state
from oracle.oracle import OracleDomain, OracleSim

pytestmark = pytest.mark.gpu

CASES = {"hartmann2d": lambda: hartmann_2d(12, 10), "duct3d": lambda: duct_3d(8, 6, 5, 2)}


def host(t):
    return t.detach().cpu().numpy()


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _setup(case, seed=0):
    dom = CASES[case]()
    dom.setAdvectionScheme(AdvectionScheme.LINEAR_UPWIND)
    seeded_state(dom, seed, scale=0.5)
    g = torch.Generator().manual_seed(seed + 10)
    for b in dom.getBlocks():
        b.setPassiveScalar(torch.rand(b.passiveScalar.shape, generator=g, dtype=torch.float64).to("cuda"))
    dom.PrepareSolve()
    return dom, OracleDomain(dom)


@pytest.mark.parametrize("case", list(CASES))
def test_linear_upwind_assembly_matches_the_oracle(cuda, case):
    dom, od = _setup(case)
    assert od.scheme == 1
    dt, nu = 0.01, float(dom.viscosity[0])
    ts = torch.tensor([dt], dtype=torch.float64)
    u = host(dom._u_block).reshape(-1)
    _C.SetupAdvectionMatrix(dom, ts, 0)
    _C.SetupAdvectionVelocity(dom, ts, 0, False)
    Cval, A = od.advection_matrix(u, dt, nu)
    central_dom = CASES[case]()
    assert rel(host(dom.C.value), Cval) < 1e-12 and rel(host(dom.A), A) < 1e-12
    assert rel(host(dom.velocityRHS), od.advection_rhs(u, None, dt, nu)) < 1e-12
    g = torch.Generator().manual_seed(3)
    ustar = torch.from_numpy(u) + 0.1 * torch.randn(u.size, generator=g, dtype=torch.float64)
    dom.velocityResult.copy_(ustar.to("cuda"))
    _C.SetupPressureCorrection(dom, ts, 0, False, False)
    assert rel(host(dom.pressureRHS), od.pressure_rhs(Cval, A, u, host(ustar), None, dt, nu)) < 1e-12
    # the scalar
    _C.SetupAdvectionMatrix(dom, ts, 0, forPassiveScalar=True, passiveScalarChannel=0)
    sval, sA = od.scalar_matrix(u, dt, nu, 0)
    assert rel(host(dom.C.value), sval) < 1e-12
    _C.SetupAdvectionScalar(dom, ts, 0)
    assert rel(host(dom.scalarRHS), od.scalar_rhs(host(dom._phi_block).reshape(-1), dt, nu, 0, u=u)) < 1e-12
    # some faces are upwinded: the matrix differs from the central one
    assert rel(Cval, OracleDomain(central_dom).advection_matrix(u, dt, nu)[0]) > 1e-6


@pytest.mark.parametrize("case", list(CASES))
def test_linear_upwind_steps_match_the_oracle(cuda, case):
    dom, od = _setup(case, seed=4)
    tol = pb.SolverTolerance(rtol=1e-12, atol=1e-14)
    ref = OracleSim(od, host(dom._u_block).reshape(-1), 0.01, float(dom.viscosity[0]), advection_tol=tol,
                    pressure_tol=tol, scalar=dict(phi=host(dom._phi_block).reshape(-1), nu=None))
    sim = pb.Simulation(dom, 0.01, non_orthogonal=False, advection_tol=tol, pressure_tol=tol)
    for _ in range(3):
        assert sim.single_step(), sim.last_error
        ref.step()
    torch.cuda.synchronize()
    assert rel(host(dom._u_block).reshape(-1), ref.u) < 1e-9
    assert rel(host(dom._phi_block).reshape(-1), ref.phi_s.reshape(-1)) < 1e-9
