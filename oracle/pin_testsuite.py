"""Pin the oracle against POT3D's own test-suite outputs -- TEST INFRASTRUCTURE.

Runs the oracle's full reference path (mesh -> Br interpolation -> RHS ->
PCG -> phi with ghosts -> energies) on the three testsuite cases, using the
fixtures written by tests/golden/make_fixtures.py, and records the results
next to the reference values in tests/golden/oracle_pin.json.

    python oracle/pin_testsuite.py [case ...]

The validator of the reference (bin/pot3d_validation.sh) compares energies
rounded to 7 decimals; the same criterion is applied here and recorded.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, ".."))
GOLD = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, HERE)

import oracle as O  # noqa: E402

CASES = ["potential_field_source_surface", "potential_field_current_sheet", "open_field"]


def load_case(case):
    with open(os.path.join(GOLD, f"{case}.json")) as fh:
        meta = json.load(fh)
    z = np.load(os.path.join(GOLD, f"{case}_br.npz"))
    return meta, z


def mesh_for(nml):
    return O.make_mesh(nml["nr"], nml["nt"], nml["np"], r0=nml["r0"], r1=nml["r1"], rfrac=nml["rfrac"],
                       drratio=nml["drratio"], nfrmesh=nml["nfrmesh"], tfrac=nml["tfrac"],
                       dtratio=nml["dtratio"], nftmesh=nml["nftmesh"], pfrac=nml["pfrac"],
                       dpratio=nml["dpratio"], nfpmesh=nml["nfpmesh"], phishift=nml["phishift"])


def br0_for(nml, mesh, z):
    return O.readbr(mesh, z["tn"], z["pn"], np.asarray(z["data"], np.float64), nml["option"],
                    nml["do_not_balance_flux"])


def validate7(a, b):
    """bin/pot3d_validation.sh: round to 7 decimals and compare."""
    return round(a, 7) == round(b, 7)


def run(case):
    meta, z = load_case(case)
    nml = meta["namelist"]
    mesh = mesh_for(nml)
    br0 = br0_for(nml, mesh, z)
    t0 = time.time()
    out = O.potfld(mesh, br0, option=nml["option"], ifprec=nml["ifprec"], epscg=nml["epscg"],
                   ncghist=nml["ncghist"])
    dt = time.time() - t0
    ref = meta["reference"]
    w = out["energy"].tolist()
    rec = {
        "iterations": out["ncg"], "ref_iterations": ref["iterations"], "epsn": out["epsn"],
        "energy": {"wr": w[0], "wt": w[1], "wp": w[2], "total": sum(w)}, "ref_energy": ref["energy"],
        "energy_match_7_decimals": all(validate7(a, ref["energy"][k]) for a, k in zip(w, ("wr", "wt", "wp"))),
        "history": out["history"], "seconds": dt, "threads": O.threads(),
    }
    return rec


def main(cases):
    path = os.path.join(GOLD, "oracle_pin.json")
    res = {}
    if os.path.exists(path):
        with open(path) as fh:
            res = json.load(fh)
    for c in cases:
        rec = run(c)
        res[c] = rec
        print(c, rec["iterations"], rec["ref_iterations"], rec["energy"], rec["energy_match_7_decimals"],
              f"{rec['seconds']:.1f}s", flush=True)
        with open(path, "w") as fh:
            json.dump(res, fh, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:] or CASES)
