"""bench.py's reference arm runs on the host alone (the reference's KernelX100 from oracle/_ref):
its one JSON line carries the contract's keys with the reference arm's conventions."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref")), reason="oracle/_ref not built")
def test_reference_arm_json_line():
    # run through runpy so the same process can list the shared objects it loaded
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--rows', '40000000', '--steps', '1', "
            "'--warmup', '0']\n"
            "try:\n    runpy.run_path('bench.py', run_name='__main__')\nexcept SystemExit:\n    pass\n"
            "print('LOADED', sorted({l.split()[-1] for l in open('/proc/self/maps') if l.rstrip().endswith('.so')}))")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    loaded = [p for p in lines[-1].split("'") if p.startswith(ROOT)]
    # the reference arm runs the reference's own code only: nothing of the product is loaded
    assert loaded and all(os.path.join("oracle", "_ref") in p for p in loaded), loaded
    line = json.loads(lines[-2])
    if "unavailable" in line:
        pytest.skip(line["unavailable"])
    assert line["impl"] == "reference"
    for k in ["metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "config",
              "cpu_baseline", "e2e"]:
        assert k in line, k
    assert line["value"] > 0 and line["higher_is_better"] is True and line["unit"] == "rows/s"
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert line["config"]["rows_per_gpu"] == 40_000_000 and "40,000,000 rows per step" in cb["sample"]
