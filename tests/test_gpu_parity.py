"""Kernel parity: every phipict_b200 assembly kernel against the CPU oracle on the same
seeded inputs, through the phiPICT-style backend functions (which call the C ABI).

Bars: float64 within 1e-12 relative (the reference's batched==single bar is 1e-9/1e-8,
tests/test_batching.py:113-174), float32 within 1e-5 relative."""
import numpy as np
import pytest
import torch

import phipict_b200 as pb
from phipict_b200 import _C
from cases import duct_3d, hartmann_2d, rotated_pair_2d, seeded_state
from oracle.oracle import OracleDomain

pytestmark = pytest.mark.gpu

CASES = {
    "hartmann2d": lambda dt: hartmann_2d(12, 10, dtype=dt),
    "duct3d": lambda dt: duct_3d(7, 6, 5, 2, dtype=dt),
    "rotated2d": lambda dt: rotated_pair_2d(6, dtype=dt),
}
RTOL = {torch.float64: 1e-12, torch.float32: 1e-5}


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def setup(case, dtype, seed=0):
    dom = CASES[case](dtype)
    seeded_state(dom, seed)
    dom.PrepareSolve()
    od = OracleDomain(dom, 0, np.float64 if dtype == torch.float64 else np.float32)
    return dom, od


def host(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("case", list(CASES))
def test_advection_and_pressure_assembly(cuda, case, dtype):
    dom, od = setup(case, dtype)
    dt, nu = 0.01, float(dom.viscosity[0])
    ts = torch.tensor([dt], dtype=torch.float64)
    u = host(dom._u_block).reshape(-1)
    # momentum matrix (PISO_build_matrix) and RHS
    _C.SetupAdvectionMatrix(dom, ts, 0)
    _C.SetupAdvectionVelocity(dom, ts, 0, False)
    Cval, A = od.advection_matrix(u, dt, nu)
    assert np.array_equal(host(dom.C.index), od.col)
    assert np.array_equal(host(dom.C.row), od.row)
    assert rel(host(dom.C.value), Cval) < RTOL[dtype]
    assert rel(host(dom.A), A) < RTOL[dtype]
    rhs = od.advection_rhs(u, None, dt, nu)
    assert rel(host(dom.velocityRHS), rhs) < RTOL[dtype]
    # pressure matrix, HbyA and divergence with a perturbed u*
    g = torch.Generator(device="cpu").manual_seed(1)
    ustar = (torch.from_numpy(u.astype(np.float64)) + 0.1 * torch.randn(u.size, generator=g, dtype=torch.float64)).to(dtype)
    dom.velocityResult.copy_(ustar.to(cuda))
    _C.SetupPressureCorrection(dom, ts, 0, False, False)
    Pval, Pcol = od.laplace_matrix(A)
    assert rel(host(dom.P.value), Pval) < RTOL[dtype]
    h = od.pressure_rhs(Cval, A, u, host(ustar), None, dt, nu)
    assert rel(host(dom.pressureRHS), h) < RTOL[dtype]
    div = od.divergence(h)
    assert rel(host(dom.pressureRHSdiv), div) < 10 * RTOL[dtype] * max(1.0, np.abs(h).max() / max(np.abs(div).max(), 1e-30))
    # velocity correction with a random pressure field
    p = torch.randn(dom.getTotalSize(), generator=g, dtype=torch.float64).to(dtype)
    dom.pressureResult.copy_(p.to(cuda))
    _C.CopyPressureResultToBlocks(dom)
    _C.CorrectVelocity(dom, ts, version=1)
    ucorr = od.correct_velocity(host(p), host(dom.pressureRHS), host(dom.A))
    assert rel(host(dom.velocityResult), ucorr) < RTOL[dtype]


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("case", ["hartmann2d", "duct3d"])
def test_potential_assembly_and_current_density(cuda, case, dtype):
    dom, od = setup(case, dtype)
    dom.SetupEpotOnDomain()
    Eval, Ecol = od.laplace_matrix(epot=True)
    assert rel(host(dom.Epot.value), Eval) < RTOL[dtype]
    d, n = dom.getSpatialDims(), dom.getTotalSize()
    g = torch.Generator(device="cpu").manual_seed(2)
    field = torch.randn(d * n, generator=g, dtype=torch.float64).to(dtype)
    rhs = _C.ComputeEpotRHS(dom, field.to(cuda))
    assert rel(host(rhs), od.epot_rhs(host(field))) < 10 * RTOL[dtype]
    phi = torch.randn(n, generator=g, dtype=torch.float64).to(dtype)
    uxb = torch.randn(3 * n, generator=g, dtype=torch.float64).to(dtype)
    J = _C.ComputeCurrentDensityFaceBased(dom, phi.to(cuda), uxb.to(cuda))
    assert rel(host(J), od.current_density(host(phi), host(uxb))) < 10 * RTOL[dtype]


def test_potential_boundary_conditions(cuda):
    """Thin-wall, Dirichlet (with values) and open faces, uniform and per-cell masks."""
    dom = duct_3d(6, 5, 4, 1, dtype=torch.float64)
    blk = dom.getBlocks()[0]
    blk.getBoundary("-y").setPotentialBC(pb.PotentialBC.THIN_WALL, cw=0.1)
    fz, fx = 4, 6
    types = torch.zeros(1, 1, fz, 1, fx, dtype=torch.int8)
    types[..., ::2] = int(pb.PotentialBC.DIRICHLET)
    types[..., 1::3] = int(pb.PotentialBC.THIN_WALL)
    blk.getBoundary("+y").setPotentialTypes(types, cw=0.2)
    g = torch.Generator().manual_seed(3)
    blk.getBoundary("+y").setPotentialValues(torch.randn(1, 1, fz, 1, fx, generator=g, dtype=torch.float64))
    dom.PrepareSolve()
    dom.SetupEpotOnDomain()
    od = OracleDomain(dom)
    Eval, _ = od.laplace_matrix(epot=True)
    assert rel(host(dom.Epot.value), Eval) < 1e-12
    n = dom.getTotalSize()
    field = torch.randn(3 * n, generator=g, dtype=torch.float64)
    assert rel(host(_C.ComputeEpotRHS(dom, field.to(cuda))), od.epot_rhs(field.numpy())) < 1e-11
    phi = torch.randn(n, generator=g, dtype=torch.float64)
    uxb = torch.randn(3 * n, generator=g, dtype=torch.float64)
    J = _C.ComputeCurrentDensityFaceBased(dom, phi.to(cuda), uxb.to(cuda))
    assert rel(host(J), od.current_density(phi.numpy(), uxb.numpy())) < 1e-11


def test_constant_dirichlet_potential_is_exact(cuda):
    """phi = c on a Dirichlet face, no u x B: E phi == rhs and J == 0
    (tests/test_potential_bc.py:455-471)."""
    c = 0.7
    dom = duct_3d(6, 5, 4, 1, dtype=torch.float64)
    bnd = dom.getBlocks()[0].getBoundary("-y")
    bnd.setPotentialBC(pb.PotentialBC.DIRICHLET)
    bnd.setPotentialValues(torch.full((1, 1, 4, 1, 6), c, dtype=torch.float64))
    dom.PrepareSolve()
    dom.SetupEpotOnDomain()
    n = dom.getTotalSize()
    zero = torch.zeros(3 * n, dtype=torch.float64, device=cuda)
    phi = torch.full((n,), c, dtype=torch.float64, device=cuda)
    rhs = _C.ComputeEpotRHS(dom, zero)
    E = torch.sparse_csr_tensor(dom.Epot.row.long(), dom.Epot.index.long(), dom.Epot.value, (n, n))
    torch.testing.assert_close(E @ phi, rhs, rtol=0, atol=1e-12)
    assert float(rhs.abs().max()) > 0
    J = _C.ComputeCurrentDensityFaceBased(dom, phi, zero)
    torch.testing.assert_close(J, torch.zeros_like(J), rtol=0, atol=1e-12)


def test_batched_assembly_matches_single(cuda):
    """B environments with different states assemble what each assembles alone."""
    B = 3
    single = []
    for b in range(B):
        dom = hartmann_2d(10, 8)
        seeded_state(dom, 10 + b)
        dom.PrepareSolve()
        _C.SetupAdvectionMatrix(dom, torch.tensor([0.01], dtype=torch.float64), 0)
        single.append(host(dom.C.value))
    dom = hartmann_2d(10, 8)
    dom.setBatchSize(B)
    dom.PrepareSolve()
    for b in range(B):
        ref = hartmann_2d(10, 8, device="cpu")
        seeded_state(ref, 10 + b)
        dom.getBlocks()[0].velocity[b].copy_(ref.getBlocks()[0].velocity[0].to(cuda))
    _C.SetupAdvectionMatrix(dom, torch.tensor([0.01], dtype=torch.float64), 0)
    vals = host(dom.C.value).reshape(B, -1)
    for b in range(B):
        assert np.array_equal(vals[b], single[b])
