"""phiPICT's own Python drivers over phipict_b200's backend: the unmodified reference package
(its Simulation / MHDSimulation and piso_diff wrappers) runs with phipict_b200 in the place of
``phipict._C`` and must reproduce the fields the complete reference computed, on the 2D
Hartmann channel (200 steps) and the 3-block MHD duct (20 steps). Each case runs in a child
process so that the reference package does not stay imported. It needs the reference package
copy made by oracle/build_ref.py (``oracle/_ref/phipict``)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
REF_PACKAGE = ROOT / "oracle" / "_ref" / "phipict"
SCRIPT = ROOT / "tests" / "golden" / "reference_driver.py"
BAR = 1e-10  # the bar of the reference fixtures (every solve at rtol 1e-14)


@pytest.mark.parametrize("case", ["c1", "c2r"])
def test_reference_driver_over_this_backend(cuda, case):
    if not (REF_PACKAGE / "__init__.py").exists():
        pytest.skip("the reference package copy (oracle/build_ref.py) is not present")
    r = subprocess.run([sys.executable, str(SCRIPT), case], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["driver"].startswith("phipict.simulation.mhd")
    assert out["domain"].startswith("phipict_b200.")
    worst = max(out["rel"].items(), key=lambda kv: kv[1])
    assert worst[1] < BAR, worst
