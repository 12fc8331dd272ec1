"""Oracle solves of the 255x361x721 PFSS workload (seed 2) -- a one-time
fixture for the parity checks of the full-size GPU solves and for the
iteration counts the CPU reference arm of bench.py projects to.

    python tests/golden/make_c2_oracle.py --ifprec 1|2 [--threads N]

Builds the case with the oracle alone (its mesh, the seeded map generator
and readbr), solves it with the oracle's cgsolve (the reference's CPU PCG,
ifprec 1 or 2) from zero to epscg 1e-11 with the residual logged at every
iteration, and writes tests/golden/pfss_255x361x721_oracle_ifprec<N>.json
(iterations to 1e-9 and to 1e-11, energies of the 1e-11 solution, seconds
per iteration) and .npz (phi on three radial surfaces, every 4th theta and
phi point; ghosts included).  A diagonal solve takes about 40 minutes on
8 cores, an ILU(0) one (sequential sweeps) over an hour.
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402

WORKLOAD = "pfss_255x361x721"
SLICE_I = (2, 128, 253)  # Fortran radial indices of the stored phi surfaces
STRIDE = 4


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ifprec", type=int, required=True, choices=[1, 2])
    ap.add_argument("--epscg", type=float, default=1e-11)
    args = ap.parse_args()
    w = O.WORKLOADS[WORKLOAD]
    t0 = time.time()
    mesh, br0 = O.pfss_case(w["nr"], w["nt"], w["np"], w["lmax"], w["nbip"], w["seed"])
    s = O.Solver(mesh, br0, option="ss", ifprec=args.ifprec)
    b = s.rhs()
    t1 = time.time()
    out = s.cgsolve(np.zeros(s.N), b, epscg=args.epscg, ncghist=1, hist_cap=1 << 16)
    t2 = time.time()
    hist = out["history"]
    n9 = next((it for it, e in hist if e < 1e-9), None)
    phi = s.finalize_phi(out["x"])
    wgy = s.energy(phi)
    sl = np.stack([phi[i - 1, ::STRIDE, ::STRIDE] for i in SLICE_I])
    stem = os.path.join(HERE, f"{WORKLOAD}_oracle_ifprec{args.ifprec}")
    np.savez_compressed(stem + ".npz", phi_slices=sl, slice_i=np.array(SLICE_I), stride=STRIDE)
    rec = {"workload": WORKLOAD, "seed": w["seed"], "ifprec": args.ifprec, "epscg": args.epscg,
           "ierr": out["ierr"], "iterations": out["ncg"], "iterations_to_1e-9": n9, "epsn": out["epsn"],
           "energy": wgy.tolist(), "setup_seconds": t1 - t0, "solve_seconds": t2 - t1,
           "seconds_per_iteration": (t2 - t1) / max(1, out["ncg"]), "threads": O.threads(),
           "cpu": platform.processor() or platform.machine(),
           "history_every_100": [[it, e] for it, e in hist if it % 100 == 0]}
    with open(stem + ".json", "w") as fh:
        json.dump(rec, fh, indent=1)
    print(json.dumps({k: v for k, v in rec.items() if k != "history_every_100"}))


if __name__ == "__main__":
    main()
