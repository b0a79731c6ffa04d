"""_C.AMGPCGSolve, the CSR AMG-preconditioned CG for callers that bring an algebraic hierarchy,
against phiPICT's own solver (ref_amg_pcg.npz, made by make_ref_fields.py --amg) and the CPU
oracle's restatement of it (oracle/amg_pcg.py) on the cases of amg_cases.py."""
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from phipict_b200 import _C
from oracle import amg_pcg as oracle

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import amg_cases as ac  # noqa: E402

pytestmark = pytest.mark.gpu
FIXTURE = Path(__file__).resolve().parent / "golden" / "ref_amg_pcg.npz"
# solution bars relative to max|x| of phiPICT's solution: float64 systems stop at the same
# iteration as phiPICT, so what remains is rounding; float32 vectors carry float32 rounding
X_BAR = {"f64": 1e-9, "f32": 2e-5}


def solve(name):
    case = ac.build(name)
    args, kw = ac.torch_args(case, torch.device("cuda"), torch)
    infos = _C.AMGPCGSolve(*args, **kw)
    return case, args[6].double().cpu().numpy().reshape(case["nenv"], -1), infos


@pytest.mark.parametrize("name", list(ac.CASES))
def test_matches_reference_solver(cuda, name):
    ref = np.load(FIXTURE)
    case, x, infos = solve(name)
    xr, ir = ref[f"{name}_x"], ref[f"{name}_info"]
    for e, info in enumerate(infos):
        assert info.converged == bool(ir[e, 2]) and info.isFiniteResidual == bool(ir[e, 3])
        if name in ac.EXACT:
            assert info.usedIterations == int(ir[e, 1])
            assert abs(info.finalResidual - ir[e, 0]) <= 1e-6 * ir[e, 0]
        else:
            assert abs(info.usedIterations - int(ir[e, 1])) <= 1
    err = np.abs(x - xr).max() / np.abs(xr).max()
    assert err < X_BAR[case["dtype"]], err


@pytest.mark.parametrize("name", list(ac.CASES))
def test_matches_oracle(cuda, name):
    case, x, infos = solve(name)
    xo, io = oracle.amg_pcg(case["A_env"], case["levels_env"], case["pinv_env"], case["b"], case["x0"],
                            **ac.oracle_kwargs(case))
    for info, o in zip(infos, io):
        assert info.converged == o.converged and info.status == o.status
        if name in ac.EXACT:
            assert info.usedIterations == o.usedIterations
            assert abs(info.finalResidual - o.finalResidual) <= 1e-6 * o.finalResidual
    if case["dtype"] == "f64" and case["hdtype"] == "f64":
        assert np.abs(x - xo).max() / np.abs(xo).max() < 1e-9


def test_non_finite_right_hand_side_stops_that_environment_only(cuda):
    case = ac.build("shared_two_rhs")
    case["b"][1, 5] = np.nan
    args, kw = ac.torch_args(case, torch.device("cuda"), torch)
    infos = _C.AMGPCGSolve(*args, **kw)
    assert infos[0].converged and infos[0].isFiniteResidual
    assert not infos[1].converged and not infos[1].isFiniteResidual and infos[1].status == oracle.NONFINITE
    assert infos[1].usedIterations == 0


def test_zero_right_hand_side_converges_without_iterating(cuda):
    case = ac.build("poisson_f64")
    case["b"][:] = 0.0
    args, kw = ac.torch_args(case, torch.device("cuda"), torch)
    infos = _C.AMGPCGSolve(*args, **kw)
    assert infos[0].converged and infos[0].usedIterations == 0 and infos[0].finalResidual == 0.0
    assert torch.count_nonzero(args[6]).item() == 0


def test_argument_errors(cuda):
    case = ac.build("batched_values")
    args, kw = ac.torch_args(case, torch.device("cuda"), torch)
    with pytest.raises(RuntimeError, match="tolerances"):
        _C.AMGPCGSolve(*args, **dict(kw, tolerances=[1e-6]))
    bad = list(args)
    bad[5] = args[5].float()
    with pytest.raises(RuntimeError, match="same dtype"):
        _C.AMGPCGSolve(*bad, **kw)
    bad = list(args)
    bad[3] = [lv[:9] for lv in args[3]]
    with pytest.raises(RuntimeError, match="each AMG level"):
        _C.AMGPCGSolve(*bad, **kw)
    bad = list(args)
    bad[4] = args[4][0]  # one shared coarse inverse is fine; a wrong size is not
    _C.AMGPCGSolve(*bad, **kw)
    bad[4] = args[4][:, :-1, :-1].contiguous()
    with pytest.raises(RuntimeError, match="do not chain|wrong size"):
        _C.AMGPCGSolve(*bad, **kw)
