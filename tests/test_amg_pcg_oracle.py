"""The CPU restatement of phiPICT's AMG-preconditioned CG (oracle/amg_pcg.py): its solutions
against SciPy's direct solver, and its iteration counts and solutions against phiPICT's own
solver run on the same cases (ref_amg_pcg.npz)."""
import sys
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from oracle import amg_pcg as oracle

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import amg_cases as ac  # noqa: E402

FIXTURE = Path(__file__).resolve().parent / "golden" / "ref_amg_pcg.npz"


def run(name):
    case = ac.build(name)
    x, infos = oracle.amg_pcg(case["A_env"], case["levels_env"], case["pinv_env"], case["b"], case["x0"],
                              **ac.oracle_kwargs(case))
    return case, x, infos


@pytest.mark.parametrize("name", [n for n in ac.CASES if n != "best_maxit"])
def test_oracle_solves_the_system(name):
    case, x, infos = run(name)
    assert all(i.converged for i in infos)
    for e in range(case["nenv"]):
        A, b = case["A_env"][e], case["b"][e]
        if ac.CASES[name]["neumann"]:
            r = (b - b.mean()) - A @ x[e]
            assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-8
            assert abs(x[e].mean()) < 1e-10 * np.abs(x[e]).max() + 1e-12
        else:
            xs = spla.spsolve(A.tocsc(), b)
            tol = case["opts"].get("tolerances", [case["opts"]["tolerance"]] * case["nenv"])[e]
            assert np.abs(x[e] - xs).max() / np.abs(xs).max() < max(1e3 * tol, 1e-9)


def test_oracle_reports_max_iterations_with_the_reference_count():
    case, x, infos = run("best_maxit")
    assert infos[0].status == oracle.MAXIT and not infos[0].converged
    assert infos[0].usedIterations == case["opts"]["maxIterations"] - 1


@pytest.mark.parametrize("name", list(ac.CASES))
def test_oracle_matches_reference_solver(name):
    if not FIXTURE.exists():
        pytest.fail("ref_amg_pcg.npz missing: run make_ref_fields.py --amg on a GPU")
    ref = np.load(FIXTURE)
    case, x, infos = run(name)
    xr, ir = ref[f"{name}_x"], ref[f"{name}_info"]
    for e, info in enumerate(infos):
        assert info.converged == bool(ir[e, 2])
        if name in ac.EXACT:
            assert info.usedIterations == int(ir[e, 1])
            assert abs(info.finalResidual - ir[e, 0]) <= 1e-6 * ir[e, 0]
    if name in ac.EXACT:
        assert np.abs(x - xr).max() / np.abs(xr).max() < 1e-9
