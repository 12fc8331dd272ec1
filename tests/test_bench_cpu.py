"""bench.py's reference arm on CPU: one JSON line with the contract's keys,
the oracle timed on the same workload (the whole solve on small grids, a
bounded sample projected to the oracle's own iteration count on large
ones), built and solved without the product library."""
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
    assert line["config"]["workload"] == "pfss_63x91x181" and line["config"]["ifprec"] == 2
    cb = line["cpu_baseline"]
    # the 63x91x181 ILU(0) solve is timed whole: the oracle's own 273 iterations
    assert cb["kind"] == "port" and cb["cores"] >= 1 and "273 iterations" in cb["sample"]
    assert line["projected"] is False and cb["iterations"] == 273
    assert cb["value"] == pytest.approx(line["value"])
    assert line["e2e"] == {"value": line["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_maps_no_product_library():
    code = ("import sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'pfss_63x91x181', "
            "'--ifprec', '1']; import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print('PRODUCT_SO', 'libpot3d_gpu' in maps, 'ORACLE_SO', 'liboracle' in maps)")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "PRODUCT_SO False ORACLE_SO True" in out.stdout


def test_reference_arm_needs_the_oracle_fixture_on_large_grids():
    out = _run("--impl", "reference", "--steps", "1", "--warmup", "0", "--workload", "pfss_127x181x361",
               "--ifprec", "2")
    assert out.returncode != 0 and "make_c2_oracle.py" in (out.stderr + out.stdout)
