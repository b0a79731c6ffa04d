"""Checkpoint and resume through the domain file pair: a run saved after two steps, loaded
into a fresh domain and continued matches the uninterrupted run (the momentum solve's warm
start is not part of the file, so the match is to the solver tolerance, not bitwise)."""
from pathlib import Path

import numpy as np
import pytest
import torch

import phipict_b200 as pb
from phipict_b200.io import load_domain, save_domain
from cases import duct_3d, seeded_state

pytestmark = pytest.mark.gpu


def test_resume_from_a_saved_domain_continues_the_run(cuda, tmp_path: Path):
    tol = pb.SolverTolerance(rtol=1e-12, atol=1e-14)

    def sim_of(dom):
        return pb.Simulation(dom, 0.01, non_orthogonal=False, advection_tol=tol, pressure_tol=tol)

    dom = duct_3d(8, 6, 5, 2)
    seeded_state(dom, 9)
    dom.getBlocks()[0].getBoundary("-x").setPassiveScalar(torch.ones(1, 1, dtype=torch.float64, device="cuda"))
    dom.PrepareSolve()
    s = sim_of(dom)
    for _ in range(2):
        assert s.single_step(), s.last_error
    save_domain(dom, tmp_path / "ck")
    for _ in range(2):
        assert s.single_step(), s.last_error
    torch.cuda.synchronize()
    resumed = load_domain(tmp_path / "ck")
    resumed.PrepareSolve()
    r = sim_of(resumed)
    for _ in range(2):
        assert r.single_step(), r.last_error
    torch.cuda.synchronize()
    for name in ("_u_block", "_p_block", "_phi_block"):
        a, b = getattr(dom, name).cpu().numpy(), getattr(resumed, name).cpu().numpy()
        assert np.abs(a - b).max() <= 1e-9 * max(np.abs(a).max(), 1e-30), name
