"""The CPU oracle against fields of phiPICT itself (no GPU needed).

The fixtures ``tests/golden/ref_*.npz`` hold the velocity, pressure and potential fields that
the reference (its own Python package and ``_C`` extension, run on a B200 by
``tests/golden/make_ref_fields.py``) produced on the configurations' seeded inputs. This pins
the oracle's restatement to the reference's outputs: the plain 2D Hartmann channel (64x32,
200 MHD PISO steps) and a reduced 3-block MHD duct (3 x 16x12x12, 20 steps), both in FP64 with
every solve to rtol 1e-14, compared at the 1e-10 relative bar of FP64 parity.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest
import torch

import phipict_b200 as pb
from oracle.oracle import OracleDomain, OracleSim

GOLD = Path(__file__).resolve().parent / "golden"
import sys  # noqa: E402

sys.path.insert(0, str(GOLD))
import ref_cases as rc  # noqa: E402

FP64_BAR = 1e-10


def load_fixture(tag: str) -> dict:
    path = GOLD / f"ref_{tag}.npz"
    if not path.exists():
        pytest.fail(f"missing reference fixture {path.name}: run tests/golden/make_ref_fields.py on a GPU")
    with np.load(path) as z:
        data = {k: z[k] for k in z.files}
    data["meta"] = json.loads(str(data["meta"]))
    return data


def flat_velocity(data: dict, step: int, nblocks: int) -> np.ndarray:
    """Block velocities [1, d, ...] of the fixture as the oracle's [d][n] vector."""
    us = [data[f"s{step}_u_{i}"][0] for i in range(nblocks)]
    d = us[0].shape[0]
    return np.concatenate([np.concatenate([u[c].ravel() for u in us]) for c in range(d)])


def flat_scalar(data: dict, key: str, step: int, nblocks: int) -> np.ndarray:
    return np.concatenate([data[f"s{step}_{key}_{i}"][0].ravel() for i in range(nblocks)])


def oracle_run(case: str, data: dict):
    """Step the oracle through the case, yielding (step, sim) at the recorded steps."""
    p = rc.C1 if case == "c1" else rc.C2R
    build = rc.build_c1 if case == "c1" else rc.build_c2r
    dom = build(pb, data, torch.float64, "cpu", prepare=False)
    od = OracleDomain(dom)
    nb = dom.getNumBlocks()
    u0 = np.concatenate([np.concatenate([data[f"velocity_{i}"][0][c].ravel() for i in range(nb)])
                         for c in range(dom.getSpatialDims())])
    tol = pb.SolverTolerance(rtol=rc.TIGHT_RTOL, atol=rc.TIGHT_ATOL)
    sim = OracleSim(od, u0, p["dt"], 1.0 / p["re"], advection_tol=tol, pressure_tol=tol,
                    mhd=dict(stuart=p["ha"] ** 2 / p["re"], e_b=[0.0, 1.0, 0.0], singular=True, potential_tol=tol))
    record = data["meta"]["record"]
    for step in range(1, max(record) + 1):
        if case == "c2r":  # the case resets the source before the Lorentz force of each step
            sim.src = None
        sim.step()
        if step in record:
            yield step, sim, nb


@pytest.mark.parametrize("case", ["c1", "c2r"])
def test_oracle_matches_reference_fields(case):
    data = load_fixture(f"{case}_fp64")
    assert data["meta"]["all_steps_ok"]
    worst = {}
    for step, sim, nb in oracle_run(case, data):
        errs = dict(u=rc.rel_l2(sim.u, flat_velocity(data, step, nb)),
                    p=rc.rel_l2(sim.p, flat_scalar(data, "p", step, nb)),
                    phi=rc.rel_l2(sim.phi, data[f"s{step}_phi"]))
        for k, e in errs.items():
            worst[k] = max(worst.get(k, 0.0), e)
        assert all(math.isfinite(e) and e < FP64_BAR for e in errs.values()), f"step {step}: {errs}"
    assert set(worst) == {"u", "p", "phi"}


def test_reference_fixture_inputs_match_generator():
    """The stored inputs are the ones the seeded generator produces (the fixture was not
    made from other inputs)."""
    for case, make in (("c1", rc.c1_inputs), ("c2r", rc.c2r_inputs)):
        data = load_fixture(f"{case}_fp64")
        for k, v in make().items():
            assert np.array_equal(np.asarray(v), data[k]), f"{case}: input {k} differs"


def test_reference_fields_are_nontrivial():
    """The pinned fields carry real dynamics: the velocity moved away from the initial state,
    the duct's potential is non-zero (in 2D with an in-plane field it vanishes), and the FP32
    run of the channel stays within 1e-5 of FP64."""
    d64 = load_fixture("c1_fp64")
    d32 = load_fixture("c1_fp32_tol1e-8")
    last = max(d64["meta"]["record"])
    u = d64[f"s{last}_u_0"]
    assert rc.rel_l2(u, d64["velocity_0"]) > 1e-4
    assert rc.rel_l2(d32[f"s{last}_u_0"], u) < 1e-5
    duct = load_fixture("c2r_fp64")
    last = max(duct["meta"]["record"])
    assert np.abs(duct[f"s{last}_phi"]).max() > 1e-3
    assert rc.rel_l2(duct[f"s{last}_u_1"], duct["velocity_1"]) > 1e-3
