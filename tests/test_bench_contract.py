"""bench.py's measurement contract, on the CPU.

* The reference arm (--impl reference) prints one JSON line with the keys the
  contract asks for (impl, value, unit, cpu_baseline of kind "port", an e2e
  object with no host<->device bytes) and never loads the GPU library: its
  inputs come from the oracle's copy of the generators.
* The phase rooflines divide the algorithmic bytes of each build phase (the
  formulas in bench.phase_rooflines' docstring) by the phase's time and by the
  HBM peak.
"""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent

RUN_REFERENCE = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--config", "lbvh64k", "--steps", "1", "--warmup", "3"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    assert not e.code, e.code
maps = open("/proc/self/maps").read()
print("LOADED_GPU_LIBRARY", "libhippie_b200" in maps)
"""


def test_reference_arm_line_and_no_gpu_library():
    out = subprocess.run([sys.executable, "-c", RUN_REFERENCE], cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    assert lines[-1] == "LOADED_GPU_LIBRARY False"
    rec = json.loads(lines[-2])
    assert rec["impl"] == "reference"
    assert rec["unit"] == "Mtris/s" and rec["value"] > 0 and rec["higher_is_better"] is True
    assert rec["steps"] == 1 and rec["warmup"] >= 3
    cb = rec["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == rec["value"] and cb["sample"]
    e2e = rec["e2e"]
    assert e2e["value"] == rec["value"] and e2e["unit"] == rec["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert rec["config"]["triangles"] == 65536 and rec["trace_mrays_s"] > 0


def test_phase_rooflines_formulas():
    sys.path.insert(0, str(ROOT))
    import bench
    n, peak = 1 << 20, 6500.0
    phases = {"boxes": [0.02], "morton": [0.01], "sort_pass": [0.01, 0.012, 0.011], "sort_segments": [0.02],
              "climb_local": [0.03], "climb": [0.01]}
    rows = {r["phase"].split(" (")[0]: r for r in bench.phase_rooflines(n, 60, phases, peak)}
    box = rows["scene box + boxes + Morton"]
    assert box["bytes"] == 36 * n + n * (12 + 36 + 8 + 4)
    srt = rows["radix sort"]
    assert srt["bytes"] == n * 8 * 2 * (8 + 4)  # 60-bit keys: eight 8-bit passes of 8-byte keys and 4-byte values
    assert srt["ms"] == pytest.approx(0.033 + 0.02)
    ref = rows["refit"]
    assert ref["bytes"] == 24 * (2 * n - 2) + 24 * (n - 1) + 8 * (n - 1) + 4 * (2 * n - 1) + 8 * (n - 1)
    assert ref["local_ms"] == pytest.approx(0.03) and ref["frontier_ms"] == pytest.approx(0.01)
    for r in rows.values():
        achieved = r["bytes"] / (r["ms"] * 1e-3) / 1e9
        assert r["achieved_gbs"] == pytest.approx(achieved, rel=1e-3)
        assert r["frac"] == pytest.approx(achieved / peak, rel=1e-3)
    # 30-bit keys are 4 bytes wide and take four passes
    rows30 = {r["phase"].split(" (")[0]: r for r in bench.phase_rooflines(n, 30, {"sort_pass": [0.01] * 4}, peak)}
    assert rows30["radix sort"]["bytes"] == n * 4 * 2 * (4 + 4)
