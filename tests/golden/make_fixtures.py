"""Generate the golden fixtures from the reference's own test suite.

Run once, in a checkout that has the POT3D sources next to it:

    python tests/golden/make_fixtures.py /path/to/POT3D

For each case of POT3D's testsuite (testsuite/<case>/input and
testsuite/<case>/reference) it writes:

* ``<case>_br.npz``  -- the input Br map (data in its stored precision, and
  its theta/phi scales), read with the project's PSI-HDF5 reader;
* ``<case>.json``    -- the namelist values the solve uses, and the reference
  run's results parsed from reference/pot3d.out: the energies
  (pot3d.out "Energy in B**2" lines), the iteration count, the convergence
  history and the printed r/t/p mesh tables.

These are input data and published outputs, not source code.  The tests read
only the files written here, never the reference tree.
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from pot3d_b200 import namelist  # noqa: E402
from pot3d_b200.psi_io import read_psi  # noqa: E402

CASES = ["potential_field_source_surface", "potential_field_current_sheet", "open_field"]
KEYS = ["nr", "nt", "np", "option", "r0", "r1", "rfrac", "drratio", "nfrmesh", "tfrac", "dtratio", "nftmesh",
        "pfrac", "dpratio", "nfpmesh", "phishift", "do_not_balance_flux", "ifprec", "epscg", "ncghist", "ncgmax",
        "br0file", "hdf32"]


def parse_out(text: str) -> dict:
    res = {}
    en = {}
    for name, key in (("Br", "wr"), ("Bt", "wt"), ("Bp", "wp")):
        m = re.search(rf"Energy in {name}\*\*2 =\s*([-+0-9.Ee]+)", text)
        en[key] = float(m.group(1))
    m = re.search(r"Magnetic energy =\s*([-+0-9.Ee]+)", text)
    en["total"] = float(m.group(1))
    res["energy"] = en
    res["energy_text"] = re.findall(r"(Energy in B[rtp]\*\*2 = \S+)", text)
    res["iterations"] = int(re.search(r"Number of iterations =\s*(\d+)", text).group(1))
    res["history"] = [[int(a), float(b)] for a, b in re.findall(r"Iteration:\s+(\d+)\s+Residual:\s+(\S+)", text)]
    tables = {}
    for lab in ("r", "t", "p"):
        m = re.search(rf"Mesh information for coordinate {lab}:.*?Mesh-point locations:\s*\n\s*i\s+{lab}\s+d{lab}\s+ratio\s*\n(.*?)\n\s*\n",
                      text, flags=re.S)
        rows = []
        for ln in m.group(1).splitlines():
            f = ln.split()
            if len(f) >= 2:
                rows.append([int(f[0]), float(f[1])])
        tables[lab] = rows
    res["mesh_tables"] = tables
    return res


def main(ref_root: str) -> None:
    for case in CASES:
        cdir = os.path.join(ref_root, "testsuite", case)
        nml = namelist.read(os.path.join(cdir, "input", "pot3d.dat"))
        vals = {k: nml.values[k] for k in KEYS}
        d = read_psi(os.path.join(cdir, "input", nml.br0file))
        np.savez_compressed(os.path.join(HERE, f"{case}_br.npz"), data=d.data, tn=d.scales[0], pn=d.scales[1])
        with open(os.path.join(cdir, "reference", "pot3d.out")) as fh:
            ref = parse_out(fh.read())
        out = {"case": case, "namelist": vals, "reference": ref,
               "source": f"testsuite/{case}/input/pot3d.dat, testsuite/{case}/reference/pot3d.out"}
        with open(os.path.join(HERE, f"{case}.json"), "w") as fh:
            json.dump(out, fh, indent=1)
        print(case, d.data.shape, d.dtype, ref["iterations"], ref["energy"])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <path of the POT3D source tree>")
    main(sys.argv[1])
