"""Batched PFSS solves over uneven grids.

The workload: n independent PFSS cases, each with its own grid drawn from
nr in {63, 95, 127}, nt in {91, 181}, np in {181, 361}, its own seeded Br map
(harmonics l <= 40, 20 bipoles) and its own source-surface radius r1 drawn
uniformly from [2, 3]; all are solved to the same ernorm tolerance by one
BatchSolver, whose kernels cover every unfinished case per launch.

    python -m pot3d_b200.batch [--n 48] [--seed 0] [--epscg 1e-9] [--ifprec 1|2]
                               [--precision fp32_refined|fp64] [--out f.json]

reports the batch time, per-case iterations and reliable updates, the
autotuner's choice and the aggregate algorithmic HBM throughput (bytes per
unknown and iteration: FP64 80 with the diagonal preconditioner and 104 with
ILU(0), FP32-inner 40 and 64), and compares with the same cases solved one
after another by the single-case solver in the same arithmetic.  The
default is the configuration's form: ILU(0), FP32-inner iterations with
FP64 reliable updates, per-case convergence.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import host
from .host import PM_R1

NR = (63, 95, 127)
NT = (91, 181)
NP = (181, 361)
LMAX, NBIP = 40, 20  # the batch's map generator: harmonics l <= 40 and 20 bipoles
BYTES_PER_UNKNOWN_ITER = {("fp64", 1): 80.0, ("fp64", 2): 104.0, ("fp32_refined", 1): 40.0,
                          ("fp32_refined", 2): 64.0}


def batch_specs(n: int = 48, seed: int = 0):
    """[(nr, nt, np, r1, br_seed)] of the uneven batch."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        out.append((int(rng.choice(NR)), int(rng.choice(NT)), int(rng.choice(NP)), float(rng.uniform(2.0, 3.0)),
                    int(seed) * 100_003 + q + 1))
    return out


def batch_cases(specs):
    """Meshes and br0 maps of the specs (PFSS grid law, source surface)."""
    meshes, brs = [], []
    for nr, nt, np_, r1, s in specs:
        mesh, br0 = host.pfss_case(nr, nt, np_, LMAX, NBIP, s, r1=r1)
        meshes.append(mesh)
        brs.append(br0)
    return meshes, brs


def main(argv=None):
    from .solver import BatchSolver, Pot3dSolver
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=48)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--epscg", type=float, default=1e-9)
    ap.add_argument("--no-sequential", action="store_true")
    ap.add_argument("--repeats", type=int, default=2)
    ap.add_argument("--out", default=None)
    ap.add_argument("--ifprec", type=int, default=2, help="1: diagonal, 2: ILU(0) (batched wavefront sweeps)")
    ap.add_argument("--precision", default="fp32_refined", choices=["fp32_refined", "fp64"])
    a = ap.parse_args(argv)
    specs = batch_specs(a.n, a.seed)
    meshes, brs = batch_cases(specs)
    unknowns = [(m.nr - 2) * (m.nt - 2) * (m.np - 2) for m in meshes]
    rep = {"n": a.n, "seed": a.seed, "epscg": a.epscg, "ifprec": a.ifprec, "precision": a.precision,
           "map": {"lmax": LMAX, "bipoles": NBIP}, "specs": specs}
    with BatchSolver(meshes, brs, [PM_R1["ss"]] * a.n, ifprec=a.ifprec, precision=a.precision) as b:
        t0 = time.perf_counter()
        (best, best_u), times = b.tune2()
        rep["tune"] = {"best_planes_per_block": best, "best_update_planes_per_block": best_u,
                       "ms": {f"{k[0]}x{k[1]}": v for k, v in times.items()}, "seconds": time.perf_counter() - t0}
        secs = []
        for _ in range(a.repeats):
            ierr = b.solve(epscg=a.epscg)
            secs.append(b.seconds)
        ncg = [i.ncg for i in b.infos]
        rep["batch"] = {"seconds": min(secs), "all_seconds": secs, "ierr": ierr, "ncg": ncg,
                        "reliable_updates": [i.n_refine for i in b.infos],
                        "kernel_launches": b.infos[0].kernel_launches}
        bpu = BYTES_PER_UNKNOWN_ITER[(a.precision, a.ifprec)]
        moved = sum(bpu * u * k for u, k in zip(unknowns, ncg))
        rep["batch"]["algorithmic_gbs"] = moved / min(secs) / 1e9
        rep["batch"]["max_case_iterations"] = max(ncg)
        sol0 = b.solution(0)
    if not a.no_sequential:
        tot, ncg1 = 0.0, []
        for q, (m, br) in enumerate(zip(meshes, brs)):
            with Pot3dSolver(m, br, ifprec=a.ifprec, precision=a.precision) as s:
                best_t = None
                for _ in range(a.repeats):
                    x = np.zeros(s.N)
                    r = s.rhs()
                    s.cgsolve(x, r, epscg=a.epscg)
                    best_t = s.last_info.seconds if best_t is None else min(best_t, s.last_info.seconds)
                tot += best_t
                ncg1.append(s.last_info.ncg)
                if q == 0:
                    rep["case0_rel_diff_vs_single"] = float(np.linalg.norm(sol0 - x) / np.linalg.norm(x))
        rep["sequential"] = {"seconds": tot, "ncg": ncg1, "algorithmic_gbs":
                             sum(bpu * u * k for u, k in zip(unknowns, ncg1)) / tot / 1e9}
        rep["speedup_vs_sequential"] = tot / rep["batch"]["seconds"]
    print(json.dumps({k: v for k, v in rep.items() if k != "specs"}))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
