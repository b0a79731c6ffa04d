"""phipict_b200.grid's cell weights against phiPICT's own grid/shapes.py make_weights
(golden outputs in tests/golden/grid_weights.json, made by tests/golden/make_grid_golden.py)."""
import json
from pathlib import Path

import numpy as np

from phipict_b200.grid import make_weights


def test_weights_match_reference():
    data = json.loads((Path(__file__).resolve().parent / "golden" / "grid_weights.json").read_text())
    assert len(data["cases"]) == 81
    for c in data["cases"]:
        got = np.asarray(make_weights(c["type"], c["res"], c["grading"], c["refinement"]))
        ref = np.asarray(c["weights"])
        assert got.shape == ref.shape and np.abs(got - ref).max() < 1e-14, c
