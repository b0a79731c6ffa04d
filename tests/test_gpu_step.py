"""Solver and full-step parity on the GPU against the CPU oracle and SciPy.

Tight solver tolerances make the step deterministic up to the solver tolerance, so the
fields of several PISO(/MHD) steps agree with the oracle's to ~1e-9 in float64
(the reference's batched-vs-single bars: 1e-9 channel, 1e-8 MHD, tests/test_batching.py)."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

import phipict_b200 as pb
from phipict_b200 import _C
from phipict_b200.solvers import BICGSTAB, CG, solver_for
from cases import duct_3d, hartmann_2d, rotated_pair_2d, seeded_state
from oracle.oracle import OracleDomain, OracleSim

pytestmark = pytest.mark.gpu

TIGHT = dict(advection_tol=pb.SolverTolerance(rtol=1e-12, atol=1e-14),
             pressure_tol=pb.SolverTolerance(rtol=1e-12, atol=1e-14))


def host(t):
    return t.detach().cpu().numpy()


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("use_graph", [0, 1, 2])
@pytest.mark.parametrize("case", ["hartmann2d", "duct3d"])
def test_pressure_cg_matches_direct_solve(cuda, case, use_graph):
    dom = hartmann_2d(14, 10) if case == "hartmann2d" else duct_3d(6, 5, 4, 2)
    seeded_state(dom, 4)
    dom.PrepareSolve()
    ts = torch.tensor([0.01], dtype=torch.float64)
    _C.SetupAdvectionMatrix(dom, ts, 0)
    _C.CopyVelocityResultFromBlocks(dom)
    _C.SetupPressureCorrection(dom, ts)
    b = dom.pressureRHSdiv.clone()
    b -= b.mean()
    x = torch.zeros_like(b)
    s = solver_for(dom, CG, torch.float64, 1, tag="t")
    tol = 1e-11
    s.solve(dom._P_st, b, x, tol, 5000, use_graph=use_graph)
    info = s.results()[0]
    assert info.converged and info.usedIterations > 0
    od = OracleDomain(dom)
    P = od.csr_matrix(host(dom.P.value))
    r = host(b) - P @ host(x)
    assert np.linalg.norm(r) / np.sqrt(r.size) < 2 * tol
    # singular pure-Neumann system: compare with a pinned direct solve after mean removal
    Pm = P.tolil()
    Pm[0, :] = 0
    Pm[0, 0] = 1
    bb = host(b).copy()
    bb[0] = 0
    ref = spla.spsolve(Pm.tocsr(), bb)
    ref -= ref.mean()
    xs = host(x) - host(x).mean()
    assert rel(xs, ref) < 1e-7


@pytest.mark.parametrize("case", ["hartmann2d", "duct3d", "rotated2d"])
def test_momentum_bicgstab_multi_rhs(cuda, case):
    dom = {"hartmann2d": lambda: hartmann_2d(12, 8), "duct3d": lambda: duct_3d(6, 5, 4, 2),
           "rotated2d": lambda: rotated_pair_2d(6)}[case]()
    seeded_state(dom, 5)
    dom.PrepareSolve()
    ts = torch.tensor([0.01], dtype=torch.float64)
    _C.SetupAdvectionMatrix(dom, ts, 0)
    _C.SetupAdvectionVelocity(dom, ts, 0, False)
    x = torch.zeros_like(dom.velocityRHS)
    d = dom.getSpatialDims()
    s = solver_for(dom, BICGSTAB, torch.float64, d, tag="t")
    s.solve(dom._C_st, dom.velocityRHS, x, 1e-12, 5000)
    infos = s.results()
    assert len(infos) == d and all(i.converged for i in infos)
    od = OracleDomain(dom)
    C = od.csr_matrix(host(dom.C.value))
    n = dom.getTotalSize()
    for k in range(d):
        ref = spla.spsolve(C, host(dom.velocityRHS)[k * n:(k + 1) * n])
        assert rel(host(x)[k * n:(k + 1) * n], ref) < 1e-9


def test_zero_rhs_and_converged_start(cuda):
    """Zero right-hand side: CG stops at once with x = 0 (tests/test_krylov.py:151-160)."""
    dom = hartmann_2d(8, 6)
    dom.PrepareSolve()
    _C.SetupAdvectionMatrix(dom, torch.tensor([0.01], dtype=torch.float64), 0)
    _C.SetupPressureMatrix(dom, torch.tensor([0.01], dtype=torch.float64))
    b = torch.zeros(dom.getTotalSize(), dtype=torch.float64, device=cuda)
    x = torch.zeros_like(b)
    s = solver_for(dom, CG, torch.float64, 1, tag="z")
    s.solve(dom._P_st, b, x, 1e-10, 100)
    info = s.results()[0]
    assert info.converged and info.usedIterations == 0
    assert float(x.abs().max()) == 0.0


def test_nonfinite_and_maxit_are_reported(cuda):
    """A NaN right-hand side is reported non-finite; maxit=1 reports max iterations
    (tests/test_krylov.py:162-180)."""
    dom = hartmann_2d(8, 6)
    seeded_state(dom, 1)
    dom.PrepareSolve()
    ts = torch.tensor([0.01], dtype=torch.float64)
    _C.SetupAdvectionMatrix(dom, ts, 0)
    _C.SetupPressureMatrix(dom, ts)
    g = torch.Generator().manual_seed(0)
    b = torch.randn(dom.getTotalSize(), generator=g, dtype=torch.float64).to(cuda)
    b -= b.mean()
    s = solver_for(dom, CG, torch.float64, 1, tag="m")
    x = torch.zeros_like(b)
    s.solve(dom._P_st, b, x, 1e-14, 1)
    info = s.results()[0]
    assert not info.converged and info.status == 3
    bn = b.clone()
    bn[3] = float("nan")
    x.zero_()
    s.solve(dom._P_st, bn, x, 1e-10, 50)
    info = s.results()[0]
    assert not info.converged and not info.isFiniteResidual


def _oracle_sim(dom, dt, mhd=None, src=None):
    od = OracleDomain(dom)
    u0 = host(dom._u_block).reshape(-1)
    return OracleSim(od, u0, dt, float(dom.viscosity[0]), advection_tol=TIGHT["advection_tol"],
                     pressure_tol=TIGHT["pressure_tol"], mhd=mhd, source=src)


@pytest.mark.parametrize("case", ["hartmann2d", "duct3d", "rotated2d"])
def test_piso_steps_match_oracle(cuda, case):
    dom = {"hartmann2d": lambda: hartmann_2d(12, 10), "duct3d": lambda: duct_3d(6, 5, 4, 2),
           "rotated2d": lambda: rotated_pair_2d(6)}[case]()
    seeded_state(dom, 7, scale=0.1)
    if case == "rotated2d":
        for b in dom.getBlocks():
            b.velocity.zero_()
    dom.PrepareSolve()
    dt = 0.01
    ref = _oracle_sim(dom, dt)
    sim = pb.Simulation(dom, dt, non_orthogonal=False, **TIGHT)
    for _ in range(3):
        assert sim.single_step()
        ref.step()
    assert rel(host(dom._u_block).reshape(-1), ref.u) < 1e-9
    assert rel(host(dom.pressureResult), ref.p) < 1e-8


@pytest.mark.parametrize("case", ["hartmann2d", "duct3d"])
def test_mhd_steps_match_oracle(cuda, case):
    dom = hartmann_2d(12, 10) if case == "hartmann2d" else duct_3d(6, 5, 4, 2)
    seeded_state(dom, 8, scale=0.1)
    dom.PrepareSolve()
    dt, N = 0.01, 2.0
    e_b = [0.0, 1.0, 0.0]
    anchored = False
    ref = _oracle_sim(dom, dt, mhd=dict(stuart=N, e_b=e_b, singular=not anchored,
                                        potential_tol=pb.SolverTolerance(rtol=1e-12, atol=1e-14)))
    sim = pb.MHDSimulation(dom, dt, torch.tensor(N), torch.tensor(e_b, dtype=torch.float64), non_orthogonal=False,
                           potential_tol=pb.SolverTolerance(rtol=1e-12, atol=1e-14), **TIGHT)
    for _ in range(3):
        assert sim.single_step()
        ref.step()
    assert rel(host(dom._u_block).reshape(-1), ref.u) < 1e-8
    assert rel(host(dom.epotResult), ref.phi) < 1e-7 or float(np.abs(ref.phi).max()) < 1e-12


def test_batched_steps_match_single(cuda):
    """B environments simulated together reproduce B separate simulations
    (tests/test_batching.py:113-127)."""
    B, steps = 3, 3
    singles = []
    for b in range(B):
        dom = hartmann_2d(10, 8)
        seeded_state(dom, 20 + b, scale=0.2)
        dom.PrepareSolve()
        sim = pb.MHDSimulation(dom, 0.01, torch.tensor(1.0), torch.tensor([0.0, 1.0, 0.0]), non_orthogonal=False, **TIGHT)
        for _ in range(steps):
            assert sim.single_step()
        singles.append(host(dom._u_block)[0])
    dom = hartmann_2d(10, 8)
    dom.setBatchSize(B)
    for b in range(B):
        ref = hartmann_2d(10, 8, device="cpu")
        seeded_state(ref, 20 + b, scale=0.2)
        dom.getBlocks()[0].velocity[b].copy_(ref.getBlocks()[0].velocity[0])
    dom.PrepareSolve()
    sim = pb.MHDSimulation(dom, 0.01, torch.tensor(1.0), torch.tensor([0.0, 1.0, 0.0]), non_orthogonal=False, **TIGHT)
    for _ in range(steps):
        assert sim.single_step()
    out = host(dom._u_block)
    for b in range(B):
        assert rel(out[b], singles[b]) < 1e-9


def test_mixed_precision_matches_fp64(cuda):
    """FP32 inner Krylov inside FP64 refinement: fields within 1e-8 of the all-FP64 step."""
    results = []
    for mixed in (False, True):
        dom = duct_3d(8, 6, 5, 2)
        seeded_state(dom, 9, scale=0.1)
        dom.PrepareSolve()
        tol = dict(advection_tol=pb.SolverTolerance(rtol=1e-11), pressure_tol=pb.SolverTolerance(rtol=1e-11))
        sim = pb.MHDSimulation(dom, 0.01, torch.tensor(2.0), torch.tensor([0.0, 1.0, 0.0]), non_orthogonal=False,
                               potential_tol=pb.SolverTolerance(rtol=1e-11), mixed_precision=mixed, **tol)
        for _ in range(3):
            assert sim.single_step()
        results.append((host(dom._u_block).copy(), host(dom.pressureResult).copy()))
    assert rel(results[1][0], results[0][0]) < 1e-8
    assert rel(results[1][1], results[0][1]) < 1e-6


@pytest.mark.parametrize("kind,nrhs", [(CG, 1), (BICGSTAB, 3)])
def test_persistent_solver_matches_graph_solver(cuda, kind, nrhs):
    """The persistent cooperative solve and the graph of per-phase kernels use the same
    per-tile arithmetic and reduction order: identical iterations and solutions."""
    dom = duct_3d(8, 6, 5, 2)
    seeded_state(dom, 13, scale=0.2)
    dom.PrepareSolve()
    ts = torch.tensor([0.01], dtype=torch.float64)
    _C.SetupAdvectionMatrix(dom, ts, 0)
    _C.SetupAdvectionVelocity(dom, ts, 0, False)
    _C.SetupPressureMatrix(dom, ts)
    if kind == CG:
        A, b = dom._P_st, dom.pressureRHSdiv.clone()
        g = torch.Generator().manual_seed(3)
        b.copy_(torch.randn(b.numel(), generator=g, dtype=torch.float64))
        b -= b.mean()
    else:
        A, b = dom._C_st, dom.velocityRHS.clone()
    out = []
    for mode in (1, 2):
        s = solver_for(dom, kind, torch.float64, nrhs, tag=f"mode{mode}")
        x = torch.zeros_like(b)
        s.solve(A, b, x, 1e-12, 5000, use_graph=mode)
        out.append((x, s.results()))
    (x1, i1), (x2, i2) = out
    assert [i.usedIterations for i in i1] == [i.usedIterations for i in i2]
    assert all(i.converged for i in i2)
    assert torch.equal(x1, x2)
