"""Run phiPICT's own Python package (its Simulation / MHDSimulation drivers, unmodified) with
phipict_b200 in the place of its compiled ``phipict._C`` module, and compare the fields with
the fixtures the complete reference produced (ref_c1_fp64.npz, ref_c2r_fp64.npz).

    python tests/golden/reference_driver.py c1|c2r [--ref-package DIR]

The reference package is the copy that oracle/build_ref.py lays next to its build
(``oracle/_ref/phipict``); its ``_C.so`` is never loaded. ``phipict._C`` becomes a module
holding phipict_b200's backend functions and classes. Reference types that phipict_b200 does
not have (VaryingDirichletBoundary, StaticDirichletBoundary, BoundarySampling and the small
index vector types) are empty classes, so the driver's isinstance checks and annotations see
no such objects. Prints one JSON line: per recorded step and field, the relative L2 distance
to the fixture.
"""
from __future__ import annotations

import argparse
import json
import sys
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

import numpy as np  # noqa: E402
import torch  # noqa: E402

STEPS = {"c1": (1, 10, 200), "c2r": (1, 5, 20)}
CLASSES = ("AdvectionScheme", "Block", "Boundary", "BoundaryConditionType", "BoundaryType", "CSRmatrix",
           "ConnectedBoundary", "ConvergenceCriterion", "Domain", "FixedBoundary", "LinearSolverResultInfo",
           "PeriodicBoundary", "PotentialBC")


def backend_module() -> types.ModuleType:
    """phipict._C made of phipict_b200's backend functions and classes."""
    import phipict_b200 as pb
    from phipict_b200 import _C as ours

    mod = types.ModuleType("phipict._C")
    for name in dir(ours):
        if not name.startswith("__"):
            setattr(mod, name, getattr(ours, name))
    for name in CLASSES:
        setattr(mod, name, getattr(pb, name))

    def absent(name):
        if name.startswith("__"):
            raise AttributeError(name)
        t = type(name, (), {})
        setattr(mod, name, t)
        return t

    mod.__getattr__ = absent
    return mod


def import_reference(package_root: Path):
    sys.modules["phipict._C"] = backend_module()
    sys.path.insert(0, str(package_root))
    import phipict

    if Path(phipict.__file__).resolve().parent != (package_root / "phipict").resolve():
        raise RuntimeError(f"imported {phipict.__file__}, not the package under {package_root}")
    return phipict


def run(case: str, package_root: Path) -> dict:
    import ref_cases as rc

    pp = import_reference(package_root)
    dev = torch.device("cuda")
    inputs = rc.c1_inputs() if case == "c1" else rc.c2r_inputs()
    dom = (rc.build_c1 if case == "c1" else rc.build_c2r)(pp, inputs, torch.float64, dev)
    sim = rc.make_sim(pp, dom, case, True)
    ref = np.load(HERE / f"ref_{case}_fp64.npz")
    out = {"case": case, "driver": type(sim).__module__ + "." + type(sim).__name__,
           "domain": type(dom).__module__ + "." + type(dom).__name__, "rel": {}}
    done = 0
    for s in STEPS[case]:
        while done < s:
            if not sim.single_step():
                raise RuntimeError(f"step {done + 1} failed")
            done += 1
        for k, v in rc.fields(dom).items():
            r = ref[f"s{s}_{k}"]
            out["rel"][f"s{s}_{k}"] = float(np.linalg.norm(v - r) / max(np.linalg.norm(r), 1e-300))
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=list(STEPS))
    ap.add_argument("--ref-package", default=str(ROOT / "oracle" / "_ref"))
    a = ap.parse_args()
    print(json.dumps(run(a.case, Path(a.ref_package))), flush=True)


if __name__ == "__main__":
    main()
