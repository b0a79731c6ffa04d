"""The solver tuner (Simulation(autotune_solvers=True)): the persistent Krylov kernels' grid
(resident CTAs per SM) is chosen per solve by measurement during the first steps. A grid
changes the launch only: per-tile partial sums are reduced in tile order whatever CTA
computed them, so every candidate gives the same bits as the default grid."""
import pytest
import torch

import phipict_b200 as pb
from phipict_b200.solvers import SolverTuner
from cases import duct_3d, hartmann_2d, seeded_state



def _run(make, autotune: bool, steps: int):
    dom = make()
    seeded_state(dom, 21, scale=0.2)
    dom.PrepareSolve()
    tol = pb.SolverTolerance(rtol=1e-10)
    sim = pb.MHDSimulation(dom, 1e-2, torch.tensor(4.0, dtype=torch.float64), torch.tensor([0.0, 1.0, 0.0]),
                           non_orthogonal=False, mixed_precision=True, pressure_use_amg=True,
                           potential_use_preconditioner=True, advection_tol=tol, pressure_tol=tol, potential_tol=tol,
                           autotune_solvers=autotune)
    if autotune:
        sim.solver_tuner.trials = 1
    for _ in range(steps):
        assert sim.single_step(), sim.last_error
    return dom, sim


@pytest.mark.gpu
@pytest.mark.parametrize("make", [lambda: duct_3d(16, 12, 12, 2), lambda: hartmann_2d(96, 64)])
def test_tuned_grids_give_the_same_bits(cuda, make):
    steps = len(SolverTuner.CANDIDATES) + 2
    d0, _ = _run(make, False, steps)
    d1, sim = _run(make, True, steps)
    rep = sim.solver_tuner.report()
    assert rep and all(v["ctas_per_sm"] in SolverTuner.CANDIDATES for v in rep.values()), rep
    assert torch.equal(d0._u_block, d1._u_block)
    assert torch.equal(d0.pressureResult, d1.pressureResult)
    assert torch.equal(d0.epotResult, d1.epotResult)


def test_tuner_picks_the_fastest_median():
    t = SolverTuner(trials=2)
    for ms in ((0, 5.0), (2, 3.0), (1, 4.0), (0, 5.5), (2, 2.5), (1, 4.5)):
        c, v = ms
        assert t.pick("p") == c
        t.record("p", c, v, 10)
    assert t.choice["p"] == 2 and t.pick("p") == 2
