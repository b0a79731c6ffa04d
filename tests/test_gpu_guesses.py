"""Extrapolated initial guesses (Simulation(extrapolate_guesses=True)): the pressure of every
corrector and the potential start from 2 x_n - x_(n-1) of the last two steps. A guess changes
only where the Krylov iteration starts, so the fields agree with the default run's to the
solver tolerance, and the solves take fewer iterations."""
import pytest
import torch

import phipict_b200 as pb
from cases import duct_3d, seeded_state

pytestmark = pytest.mark.gpu


def _run(extrapolate: bool, steps: int = 8):
    dom = duct_3d(16, 12, 12, 2)
    seeded_state(dom, 31, scale=0.2)
    dom.PrepareSolve()
    tol = pb.SolverTolerance(rtol=1e-10)
    sim = pb.MHDSimulation(dom, 1e-2, torch.tensor(4.0, dtype=torch.float64), torch.tensor([0.0, 1.0, 0.0]),
                           non_orthogonal=False, mixed_precision=True, pressure_use_amg=True,
                           potential_use_preconditioner=True, advection_tol=tol, pressure_tol=tol, potential_tol=tol,
                           pressure_warm_start=True, extrapolate_guesses=extrapolate)
    its = 0
    for _ in range(steps):
        assert sim.single_step(), sim.last_error
        its += sum(max(i.innerIterations for i in infos) for tag, infos in sim.solve_report() if tag != "velocity")
    return dom, its


def test_extrapolated_guesses_keep_the_fields(cuda):
    d0, its0 = _run(False)
    d1, its1 = _run(True)
    for a, b in ((d0._u_block, d1._u_block), (d0.pressureResult, d1.pressureResult), (d0.epotResult, d1.epotResult)):
        assert float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(a)) < 1e-8
    assert its1 < its0, (its0, its1)
