"""bench.py's reference arm on CPU: one JSON line with the contract's keys,
the oracle timed on a bounded sample and projected to a whole solve."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def _run(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    return out


def test_reference_arm_json_line():
    out = _run("--impl", "reference", "--steps", "1", "--warmup", "0", "--workload", "pfss_63x91x181")
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "s" and line["higher_is_better"] is False
    assert line["config"]["workload"] == "pfss_63x91x181"
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and "273 iterations" in cb["sample"]
    assert cb["value"] == pytest.approx(line["value"])
    assert line["e2e"] == {"value": line["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_needs_an_iteration_count():
    out = _run("--impl", "reference", "--steps", "1", "--warmup", "0", "--workload", "pfss_127x181x361",
               "--ifprec", "2")
    assert out.returncode != 0 and "--ref-iterations" in (out.stderr + out.stdout)
