"""Generates tolerance.json: outputs of phiPICT's own solvers/tolerance.py on seeded inputs.

The reference module depends on torch only, so it is loaded straight from its source file
(no package import, which would need the reference's compiled extension). Cases whose
resolution falls through to the dtype default (a zero right-hand side with no atol) are left
out: that branch imports the reference's core.piso_diff, which needs the extension; the
default values themselves (1e-5 float32, 1e-8 float64) are pinned from
core/piso_diff.py:397-421 in the test.

Run from the repository root:  python tests/golden/make_tolerance_golden.py <reference root>
(or with the root in the PHIPICT_REFERENCE environment variable)
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys

import torch

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference(root: str):
    path = os.path.join(root, "src", "phipict", "solvers", "tolerance.py")
    spec = importlib.util.spec_from_file_location("reference_tolerance", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # dataclasses look their module up there
    spec.loader.exec_module(mod)
    return mod


def rhs_cases():
    """Seeded right-hand sides: (name, dtype, tensor, batch sizes that divide it)."""
    g = torch.Generator().manual_seed(1234)
    out = []
    for dtype in (torch.float32, torch.float64):
        dn = str(dtype).replace("torch.", "")
        out.append((f"normal_512_{dn}", torch.randn(512, generator=g, dtype=torch.float64).to(dtype), [1, 2, 4, 8]))
        out.append((f"scaled_1024_{dn}", (1e3 * torch.randn(1024, generator=g, dtype=torch.float64)).to(dtype), [1, 4, 16]))
        out.append((f"tiny_333_{dn}", (1e-9 * torch.rand(333, generator=g, dtype=torch.float64)).to(dtype), [1, 3, 9]))
        x = torch.randn(3, 256, generator=g, dtype=torch.float64)
        x[1] = 0.0  # one environment at rest
        out.append((f"one_env_zero_{dn}", x.reshape(-1).to(dtype), [3]))
        out.append((f"constant_1000_{dn}", torch.full((1000,), 3.0, dtype=dtype), [1, 10]))
    return out


TOLS = [dict(rtol=1e-6), dict(rtol=1e-12, atol=1e-9), dict(atol=1e-7), dict(rtol=1e-10), dict(rtol=1e-3, atol=1e-30),
        dict(rtol=1e-20)]


def main(root: str) -> None:
    ref = load_reference(root)
    cases = []
    for name, rhs, batches in rhs_cases():
        entry = {"name": name, "dtype": str(rhs.dtype).replace("torch.", ""), "values": rhs.to(torch.float64).tolist(),
                 "rhs_scale": ref.rhs_scale(rhs), "resolved": []}
        for kw in TOLS:
            tol = ref.SolverTolerance(**kw)
            for b in batches:
                slices = rhs.reshape(b, -1).to(torch.float64)
                if kw.get("atol") is None and bool((slices.norm(dim=1) == 0).any()):
                    continue  # the dtype-default branch (see the module docstring)
                got = ref.resolve_tolerance(tol, rhs, batch_size=b)
                entry["resolved"].append({"tol": kw, "batch_size": b, "result": got})
        cases.append(entry)
    strings = [{"tol": kw, "str": str(ref.SolverTolerance(**kw))} for kw in TOLS]
    parse = []
    for spec in [None, 1e-6, 3, 2.5e-11, {"rtol": 1e-6}, {"rtol": 1e-6, "atol": 1e-12}, {"atol": 1e-9}, {"rtol": 2}]:
        r = ref.parse_tolerance(spec)
        parse.append({"spec": spec, "result": None if r is None else (r if isinstance(r, float) else {"rtol": r.rtol, "atol": r.atol})})
    errors = []
    for spec, label in [({"foo": 1.0}, "mapping with unknown keys"), ("1e-6", "string"), (True, "bool"), ([1e-6], "list")]:
        try:
            ref.parse_tolerance(spec)
            errors.append({"spec": label, "error": None})
        except Exception as e:  # noqa: BLE001 - the exception type is the golden value
            errors.append({"spec": label, "error": type(e).__name__})
    ctor = []
    for kw in [dict(), dict(rtol=0.0), dict(atol=-1.0), dict(rtol="1e-6")]:
        try:
            ref.SolverTolerance(**kw)
            ctor.append({"kwargs": kw, "error": None})
        except Exception as e:  # noqa: BLE001
            ctor.append({"kwargs": kw, "error": type(e).__name__})
    adj = []
    for v in [1e-6, 0.0, -1.0]:
        try:
            ref.set_adjoint_rtol(v)
            adj.append({"rtol": v, "error": None, "get": ref.get_adjoint_rtol()})
        except Exception as e:  # noqa: BLE001
            adj.append({"rtol": v, "error": type(e).__name__})
    ref.set_adjoint_rtol(None)
    out = {"source": "phiPICT src/phipict/solvers/tolerance.py", "precision_floor_factor": ref.PRECISION_FLOOR_FACTOR,
           "adjoint_rtol_fallback": ref.ADJOINT_RTOL_FALLBACK, "cases": cases, "str": strings, "parse": parse,
           "parse_errors": errors, "constructor_errors": ctor, "adjoint_rtol": adj}
    with open(os.path.join(HERE, "tolerance.json"), "w") as f:
        json.dump(out, f, indent=None, separators=(",", ":"))
    print(f"wrote {len(cases)} right-hand sides, {sum(len(c['resolved']) for c in cases)} resolutions")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PHIPICT_REFERENCE")
    if not root:
        sys.exit("give the reference root as the argument or in PHIPICT_REFERENCE")
    main(root)
