"""Extrapolated initial guesses (Simulation(extrapolate_guesses=True)): the pressure of every
corrector and the potential start from 2 x_n - x_(n-1) of the last two steps. A guess changes
only where the Krylov iteration starts, so the fields agree with the default run's to the
solver tolerance, and the solves take fewer iterations."""
import pytest
import torch

import phipict_b200 as pb
from cases import duct_3d, seeded_state


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


@pytest.mark.gpu
def test_extrapolated_guesses_keep_the_fields(cuda):
    d0, its0 = _run(False)
    d1, its1 = _run(True)
    for a, b in ((d0._u_block, d1._u_block), (d0.pressureResult, d1.pressureResult), (d0.epotResult, d1.epotResult)):
        assert float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(a)) < 1e-8
    assert its1 < its0, (its0, its1)


def test_extrapolation_reproduces_polynomials():
    """Order m extrapolates a polynomial of degree m in the step index exactly."""
    from phipict_b200.simulation import extrapolate_into, push_history

    for m in (1, 2, 3):
        f = lambda t: 1.0 + 2.0 * t + (0.5 * t * t if m >= 2 else 0.0) + (0.1 * t ** 3 if m >= 3 else 0.0)  # noqa: E731
        hist = []
        x = torch.zeros(1, dtype=torch.float64)
        for t in range(4):
            if t:
                push_history(hist, x, m)
            x = torch.tensor([f(t)], dtype=torch.float64)
        g = x.clone()
        extrapolate_into(g, hist, m)
        assert abs(float(g) - f(4)) < 1e-12, (m, float(g), f(4))


def test_adaptive_order_follows_the_sequence():
    """The adaptive extrapolator's degrees agree with the binomial formula and it picks the
    lowest degree that predicts the last result exactly (ties go to the lower degree)."""
    from phipict_b200.simulation import GuessExtrapolator, extrapolate_into

    ex = GuessExtrapolator(4, adaptive=True)
    seq = [torch.tensor([float(t * t), 3.0 - t * t], dtype=torch.float64) for t in range(8)]
    x = torch.zeros(2, dtype=torch.float64)
    for t, v in enumerate(seq):
        ex.guess(x)
        ex.update(v)
    assert ex.guess(x) and ex.order == 2, ex.order
    assert torch.equal(x, torch.tensor([64.0, 3.0 - 64.0], dtype=torch.float64))
    # backward-difference degrees (the comparison) against the binomial formula (the guess)
    hist = [torch.tensor([float(k) ** 3 + 0.5 * k]) for k in (6, 5, 4, 3)]
    last = torch.tensor([7.0 ** 3 + 3.5])
    ex = GuessExtrapolator(4, adaptive=True)
    ex.last, ex.hist = last.clone(), [h.clone() for h in hist]
    ex._compare(torch.zeros(1, dtype=last.dtype))
    errs = ex._errs[0]
    for m in range(5):
        g = last.clone()
        extrapolate_into(g, hist, m)
        assert abs(float(errs[m]) - abs(float(g))) < 1e-9, (m, float(errs[m]), float(g))
    # an alternating sequence is predicted best by the last value alone
    ex = GuessExtrapolator(4, adaptive=True)
    for t in range(8):
        ex.guess(x)
        ex.update(torch.tensor([1.0 + 0.01 * (-1) ** t, 0.0], dtype=torch.float64))
    ex.guess(x)
    assert ex.order == 0, ex.order
