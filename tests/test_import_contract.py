"""Import contract (the reference keeps one too, tests/test_import_contract.py:16-30): importing
the package is cheap and has no side effects — no PyTorch, SciPy or CUDA library load, no device
touched, and never the oracle.  Checked in a fresh interpreter so that nothing imported by other
tests hides a violation."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

PROBE = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import msc_b200
from msc_b200 import pp, neighbors, synth, _lib
print(json.dumps({
    "heavy": [m for m in ("torch", "scipy", "scipy.sparse", "oracle", "triton")
              if m in sys.modules],
    "lib_loaded": _lib._lib is not None,
    "api": [n for n in ("neighbors", "connectivities") if hasattr(pp, n)],
}))
"""


def test_import_is_light_and_side_effect_free():
    out = subprocess.run([sys.executable, "-c", PROBE, str(ROOT / "metal-singlecell_b200")],
                         capture_output=True, text=True, timeout=120, check=True).stdout
    r = json.loads(out.strip().splitlines()[-1])
    assert r["heavy"] == []
    assert r["lib_loaded"] is False
    assert r["api"] == ["neighbors", "connectivities"]
