"""The analytic Hartmann profile reproduced on the GPU path.

The channel of phiPICT's example and validation runs (examples/hartmann.py;
runscripts/validation/validation.py with configs/validation.yaml and case/hartmann_10.yaml):
[0, 10] x [-1, 1], 100 x 50 cells graded towards both walls (simpleGrading 10), periodic in x,
no-slip insulating walls, e_b = (0, 1, 0), Re 2, Ha 10 (N = Ha^2/Re = 50), dt 5e-3 with
adaptive substeps, a divergence-free start. Two drives:
- the example's: a uniform source G = N reset before every velocity setup, 1000 steps;
  profile u(y) = G/N (1 - cosh(Ha y)/cosh(Ha));
- the validation's: the source follows the mean velocity towards U = 1 (forcing += 0.1 (U -
  mean u_x) every step) for the case's 20000 steps (its convergence test compares with the
  initial velocity, validation.py:692-703, so the run takes max_steps), with the validation's
  tolerances; profile u(y) = U (cosh(Ha) - cosh(Ha y)) /
  (cosh(Ha) - sinh(Ha)/Ha). phiPICT's paper reports its error, mean |u - u_exact| over the
  profile / max |u_exact|, as 0.03 % for this case (paper/tables/hartmann_error_table.tex:6,
  the metric of runscripts/validation/eval_base.py:597-611).
"""
import math

import numpy as np
import pytest
import torch

import phipict_b200 as pb
from phipict_b200.grid import cell_centers, make_weights, rectilinear_vertices, span

pytestmark = pytest.mark.gpu

HA, RE = 10.0, 2.0


def hartmann_channel(nx=100, ny=50, length=10.0, re=RE, dtype=torch.float64):
    ys = span(-1.0, 1.0, make_weights("simple", ny, 10.0, "BOTH"))
    xs = [length * i / nx for i in range(nx + 1)]
    dom = pb.Domain(2, torch.tensor([1.0 / re], dtype=dtype), name="Hartmann", device="cuda", dtype=dtype)
    b = dom.CreateBlock(vertexCoordinates=rectilinear_vertices(xs, ys, dtype=dtype).cuda(), name="Block")
    b.CloseBoundary("-y")
    b.CloseBoundary("+y")
    b.MakePeriodic("x")
    dom.PrepareSolve()
    return dom


def profile_errors(block, exact_fn):
    y = cell_centers(block.vertexCoordinates.cpu())[1, :, 0].numpy()
    u = block.velocity[0, 0].mean(dim=-1).detach().cpu().numpy()
    exact = exact_fn(y)
    scale = np.abs(exact).max()
    return float(np.abs(u - exact).mean() / scale), float(np.abs(u - exact).max() / scale)


def test_example_hartmann_profile(cuda):
    dtype = torch.float64
    dom = hartmann_channel()
    block = dom.getBlocks()[0]
    stuart = HA * HA / RE
    gradient = stuart

    def apply_forcing(domain, **kwargs):
        domain.getBlocks()[0].setVelocitySource(torch.tensor([[gradient, 0.0]], dtype=dtype, device="cuda"))
        domain.UpdateDomainData()

    sim = pb.MHDSimulation(domain=dom, dt=5e-3, stuart_number=torch.tensor(stuart),
                           e_b=torch.tensor([0.0, 1.0, 0.0], dtype=dtype), substeps="ADAPTIVE", non_orthogonal=False,
                           hooks=pb.Hooks().append(pb.Hook.PRE_VELOCITY_SETUP, apply_forcing),
                           pressure_tol=pb.SolverTolerance(rtol=1e-6, atol=1e-14),
                           potential_tol=pb.SolverTolerance(rtol=1e-8, atol=1e-14))
    sim.make_divergence_free()
    for _ in range(1000):
        assert sim.single_step()
    mean_err, max_err = profile_errors(block, lambda y: gradient / stuart * (1 - np.cosh(HA * y) / math.cosh(HA)))
    print(f"example, Ha={HA}: error {100 * mean_err:.3f} % (published 0.03 %), max error {100 * max_err:.3f} %")
    assert mean_err < 3e-4 and max_err < 2e-3


def test_validation_hartmann_error(cuda):
    dtype = torch.float64
    dom = hartmann_channel()
    block = dom.getBlocks()[0]
    v = block.vertexCoordinates[0].cpu().numpy()
    area = torch.as_tensor(np.diff(v[0][0])[None, :] * np.diff(v[1][:, 0])[:, None], device="cuda")
    forcing = [1.0]  # -pressure_gradient of case/hartmann_0.yaml

    def apply_forcing(domain, **kwargs):
        u = domain.getBlocks()[0].velocity[0, 0]
        mean = float((u * area).sum() / area.sum())
        forcing[0] += 0.1 * (1.0 - mean)
        domain.getBlocks()[0].setVelocitySource(torch.tensor([[forcing[0], 0.0]], dtype=dtype, device="cuda"))
        domain.UpdateDomainData()

    rel = lambda r: pb.SolverTolerance(rtol=r, atol=1e-14)
    sim = pb.MHDSimulation(domain=dom, dt=5e-3, stuart_number=torch.tensor(HA * HA / RE),
                           e_b=torch.tensor([0.0, 1.0, 0.0], dtype=dtype), substeps="ADAPTIVE", non_orthogonal=False,
                           hooks=pb.Hooks().append(pb.Hook.PRE_VELOCITY_SETUP, apply_forcing),
                           advection_tol=1e-7, pressure_tol=rel(1e-2), pressure_tol_intermediate=rel(1e-1),
                           potential_tol=rel(1e-4), pressure_warm_start=True, adaptive_CFL=0.8)
    sim.linear_solve_max_iterations = 5000
    sim.make_divergence_free()
    steps = 20000
    for _ in range(steps):
        sim.single_step()
    exact = lambda y: (np.cosh(HA) - np.cosh(HA * y)) / (np.cosh(HA) - np.sinh(HA) / HA)
    mean_err, max_err = profile_errors(block, exact)
    print(f"validation, Ha={HA}: {steps} steps, forcing {forcing[0]:.6f}, "
          f"error {100 * mean_err:.3f} % (published 0.03 %), max {100 * max_err:.3f} %")
    assert mean_err < 5e-4
