"""bench.py's reference arm on the CPU (no GPU needed): the JSON line the
driver reads (metric, unit, value, the e2e and cpu_baseline objects, the
workload config), on a small grid, and a clear error for a grid too small
for the headline workload's TFSF inset."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def _run(*args):
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                          capture_output=True, text=True, timeout=300, cwd=ROOT)


def test_reference_arm_json_line():
    r = _run("--n", "32", "--steps", "2", "--warmup", "1", "--ref-timesteps", "1")
    assert r.returncode == 0, r.stderr
    line = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(line) == 1
    d = json.loads(line[0])
    assert d["impl"] == "reference" and d["unit"] == "MCells/s" and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 1 and d["value"] > 0
    assert d["e2e"] == {"value": d["value"], "unit": "MCells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    assert d["config"]["cells"] == 32 ** 3 and d["config"]["timesteps_per_step"] == 1


def test_reference_arm_rejects_a_grid_inside_the_inset():
    r = _run("--n", "24", "--steps", "1", "--warmup", "1")
    assert r.returncode != 0 and "TFSF inset" in r.stderr
