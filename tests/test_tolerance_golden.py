"""SolverTolerance, rhs_scale, resolve_tolerance and parse_tolerance against outputs of
phiPICT's own solvers/tolerance.py (fixture tests/golden/tolerance.json, made by
tests/golden/make_tolerance_golden.py), plus the dtype defaults of
core/piso_diff.py:397-421 for a right-hand side at rest."""
import json
import os

import pytest
import torch

from phipict_b200 import tolerance as tl

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "tolerance.json")))
DTYPES = {"float32": torch.float32, "float64": torch.float64}


def _rhs(case):
    return torch.tensor(case["values"], dtype=torch.float64).to(DTYPES[case["dtype"]])


@pytest.mark.parametrize("case", GOLDEN["cases"], ids=[c["name"] for c in GOLDEN["cases"]])
def test_resolution_matches_the_reference(case):
    rhs = _rhs(case)
    assert tl.rhs_scale(rhs) == case["rhs_scale"]
    assert case["resolved"]
    for r in case["resolved"]:
        got = tl.resolve_tolerance(tl.SolverTolerance(**r["tol"]), rhs, batch_size=r["batch_size"])
        assert got == r["result"], (r["tol"], r["batch_size"])


def test_constants_string_and_parse():
    assert tl.PRECISION_FLOOR_FACTOR == GOLDEN["precision_floor_factor"]
    assert tl.ADJOINT_RTOL_FALLBACK == GOLDEN["adjoint_rtol_fallback"]
    for s in GOLDEN["str"]:
        assert str(tl.SolverTolerance(**s["tol"])) == s["str"]
    for p in GOLDEN["parse"]:
        got = tl.parse_tolerance(p["spec"])
        if p["result"] is None or isinstance(p["result"], float):
            assert got == p["result"] and type(got) is type(p["result"])
        else:
            assert isinstance(got, tl.SolverTolerance) and (got.rtol, got.atol) == (p["result"]["rtol"], p["result"]["atol"])


def test_errors_match_the_reference():
    specs = {"mapping with unknown keys": {"foo": 1.0}, "string": "1e-6", "bool": True, "list": [1e-6]}
    errors = {"ValueError": ValueError, "TypeError": TypeError}
    for e in GOLDEN["parse_errors"]:
        with pytest.raises(errors[e["error"]]):
            tl.parse_tolerance(specs[e["spec"]])
    for e in GOLDEN["constructor_errors"]:
        with pytest.raises(errors[e["error"]]):
            tl.SolverTolerance(**e["kwargs"])
    for e in GOLDEN["adjoint_rtol"]:
        if e["error"] is None:
            tl.set_adjoint_rtol(e["rtol"])
            assert tl.get_adjoint_rtol() == e["get"]
        else:
            with pytest.raises(ValueError):
                tl.set_adjoint_rtol(e["rtol"])
    tl.set_adjoint_rtol(None)


@pytest.mark.parametrize("dtype,default", [(torch.float32, 1e-5), (torch.float64, 1e-8)])
def test_right_hand_side_at_rest_falls_back_to_the_dtype_default(dtype, default):
    assert tl.SolverTolerance(rtol=1e-6).resolve(torch.zeros(64, dtype=dtype)) == default
    assert tl.SolverTolerance(rtol=1e-6).resolve(torch.zeros(0, dtype=dtype)) == default
    x = torch.ones(3, 16, dtype=dtype)
    x[1] = 0
    got = tl.SolverTolerance(rtol=1e-6).resolve_batched(x.reshape(-1), 3)
    assert got[1] == default and got[0] == got[2] == pytest.approx(1e-6)
