"""Generates grid_weights.json: the cell weights of phiPICT's own grid/shapes.py
(``make_weights``, simpleGrading and tanh, every refinement) on a set of resolutions and
gradings, to pin phipict_b200.grid against.

shapes.py imports the reference package (and with it the compiled extension), so this runs
with the reference importable, e.g. after ``python -m oracle.build_ref``:

    PYTHONPATH=oracle/_ref python tests/golden/make_grid_golden.py
"""
from __future__ import annotations

import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = [("simple", r, g, ref) for r in (7, 12, 32, 48, 50, 51) for g in (1.0, 2.0, 10.0) for ref in ("START", "END", "BOTH")]
CASES += [("tanh", r, g, ref) for r in (12, 48, 50) for g in (0.0, 1.5, 2.0) for ref in ("START", "END", "BOTH")]


def main() -> None:
    from phipict.grid import shapes

    out = [dict(type=t, res=r, grading=g, refinement=ref, weights=[float(w) for w in shapes.make_weights(t, r, g, ref)])
           for t, r, g, ref in CASES]
    with open(os.path.join(HERE, "grid_weights.json"), "w") as f:
        json.dump({"source": "phiPICT src/phipict/grid/shapes.py make_weights", "cases": out}, f)
    print(f"wrote {len(out)} weight lists")


if __name__ == "__main__":
    main()
