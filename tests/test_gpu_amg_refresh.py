"""The pressure multigrid's refresh schedule (phiPICT's coarse_refresh_interval,
core/piso_simulation.py:1042-1046,2268-2297,2376-2392): the whole hierarchy is set up on
every 4th change of the pressure matrix and when a solve marked its coarse operators stale;
in between only the finest level's smoother follows the matrix. A staler preconditioner only
changes where CG goes on its way to the tolerance, so the fields agree with full setups on
every step."""
from types import SimpleNamespace

import pytest
import torch

import phipict_b200 as pb
from cases import duct_3d, seeded_state
from phipict_b200.amg import AmgHierarchy


def test_stale_rule_follows_the_reference():
    h = SimpleNamespace(refreshes=1, baseline_iterations=None, stale=False)
    AmgHierarchy.note_iterations(h, 20)  # the solves right after a full setup set the baseline
    AmgHierarchy.note_iterations(h, 24)
    assert h.baseline_iterations == 24 and not h.stale
    h.refreshes = 2
    AmgHierarchy.note_iterations(h, 2 * 24 + 5)  # at the limit: not stale
    assert not h.stale and h.baseline_iterations == 24
    AmgHierarchy.note_iterations(h, 2 * 24 + 6)
    assert h.stale


def _run(interval: int, steps: int = 6):
    dom = duct_3d(16, 12, 12, 2)
    seeded_state(dom, 31, scale=0.2)
    dom.PrepareSolve()
    tol = pb.SolverTolerance(rtol=1e-10)
    sim = pb.MHDSimulation(dom, 1e-2, torch.tensor(4.0, dtype=torch.float64), torch.tensor([0.0, 1.0, 0.0]),
                           non_orthogonal=False, mixed_precision=True, pressure_use_amg=True,
                           potential_use_preconditioner=True, advection_tol=tol, pressure_tol=tol, potential_tol=tol,
                           pressure_amg_options={"coarse_refresh_interval": interval})
    for _ in range(steps):
        assert sim.single_step(), sim.last_error
    return dom, sim._amg_cache["P"]


@pytest.mark.gpu
def test_refresh_interval_keeps_the_fields(cuda):
    d1, h1 = _run(1)
    d4, h4 = _run(4)
    assert h1.full_setups == 6
    assert h4.full_setups == 2, h4.full_setups  # steps 1 and 5
    for a, b in ((d1._u_block, d4._u_block), (d1.pressureResult, d4.pressureResult), (d1.epotResult, d4.epotResult)):
        assert float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(a)) < 1e-8
