"""Benchmark: seconds to solve POT3D's PCG to epsn <= 1e-9 on one B200.

One step = one complete PCG solve of the PFSS workload 255x361x721 (65.3 M
unknowns, seeded synthetic Br: spherical harmonics l<=40 plus 20 bipoles),
from a zero guess to the reference's stopping rule epsn < epscg = 1e-9
(ernorm, src/pot3d.F90:4430-4433).  The default solver is the reference's
ILU(0) preconditioner (ifprec=2) applied in FP32 by the wavefront sweeps
inside FP64 PCG; the plain FP64 PCG with the diagonal preconditioner
(ifprec=1, the reference's default) is timed in the same run and reported
beside it (`plain_fp64`).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME] [--ifprec 1|2] [--precision fp64|fp32_refined]
                    [--no-plain]

value: device time of the solve (CUDA events on the library's stream around
the PCG initialisation and iterations), inputs resident in HBM.
e2e: the same solve through the C-ABI with pinned host buffers,
pot3d_gpu_cgsolve, host<->device copies of x and r included, wall time.
The working set (~2.6 GB of vectors, plus ~2.5 GB of sweep coefficient
streams with ILU(0)) is 20x the 126 MB L2, so no flush is needed between
steps.

Multi-GPU: replicas only (each rank solves its own instance); the reported
time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solve s to 1e-9 resid: learned+FP32-refined vs plain FP64 PCG on 1 B200; HBM GB/s"
# Iteration counts of the seeded workloads' solves from a zero guess (FP64
# PCG to 1e-9; (workload, ifprec) -> iterations), used to project the
# reference arm's CPU sample to a whole solve: the GPU solves' counts, and
# for the two smaller grids the oracle's full solves.
SOLVE_ITERATIONS = {("pfss_255x361x721", 1): 7036, ("pfss_255x361x721", 2): 1094,
                    ("pfss_63x91x181", 1): 1302, ("pfss_63x91x181", 2): 273,
                    ("pfss_127x181x361", 1): 3064,
                    ("open_511x721x1441", 1): 15639, ("open_511x721x1441", 2): 2165}
# Algorithmic DRAM bytes per unknown and PCG iteration: diagonal
# preconditioner 80 (stencil r, p -> p, Ap; update x, p, r, Ap -> x, r);
# ILU(0) 136 (stencil p, z32 -> p, Ap: 28; update x, p, r, Ap -> x, r, r32:
# 52; forward sweep r32, 3 coefficients -> y: 20; backward sweep y, 3
# coefficients + dinv -> z32: 24; r.z: 12).
BYTES_PER_UNKNOWN_ITER = {1: 80.0, 2: 136.0}
SWEEP_BYTES_PER_UNKNOWN = {"k_dilu_wave<fwd>": 20.0, "k_dilu_wave<bwd>": 24.0}
FALLBACK_HBM_GBS = 6650.0


def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def measured_traffic(kernel: str, workload: str):
    """Per-launch DRAM bytes of a kernel on a workload from the committed ncu
    summary (profiles/ncu_traffic.txt: 'kernel workload bytes_per_launch'),
    or None."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(p):
        return None
    for ln in open(p):
        f = ln.split()
        if len(f) >= 3 and f[0] == kernel and f[1] == workload and not ln.startswith("#"):
            try:
                return float(f[2])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.rows.append([x.strip() for x in ln.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def build_case(name: str, rank: int = 0):
    from pot3d_b200 import host
    w = dict(host.WORKLOADS[name])
    opt = w.pop("option", "ss")
    dnb = w.pop("do_not_balance_flux", False)
    seed = replica_seed(w.pop("seed"), rank)
    mesh, br0 = host.pfss_case(w["nr"], w["nt"], w["np"], w["lmax"], w["nbip"], seed, option=opt,
                               do_not_balance_flux=dnb)
    return mesh, br0, opt, seed


def cpu_baseline(mesh, br0, option, ifprec, ncg_target, sample_iters):
    """The oracle (CPU restatement of the reference's PCG, OpenMP on the
    host cores) timed on a bounded sample of the same workload: set-up, RHS
    and `sample_iters` PCG iterations; the solve time is projected to the
    iteration count the full solve needs."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    mo = O.Mesh(mesh.nr, mesh.nt, mesh.np, *[getattr(mesh, f) for f in O.MESH_FIELDS])
    t0 = time.perf_counter()
    s = O.Solver(mo, br0, option, ifprec)
    b = s.rhs()
    t1 = time.perf_counter()
    out = s.cgsolve(np.zeros(s.N), b, ncgmax=sample_iters, epscg=0.0)
    t2 = time.perf_counter()
    per_it = (t2 - t1) / max(1, out["ncg"])
    del s
    return {"value": per_it * ncg_target, "unit": "s", "cores": O.threads(), "kind": "port",
            "sample": f"oracle PCG set-up + {out['ncg']} iterations on {mesh.nr}x{mesh.nt}x{mesh.np}, "
                      f"{per_it * 1e3:.1f} ms/iteration, projected to {ncg_target} iterations "
                      f"(set-up {t1 - t0:.1f} s not included)",
            "seconds_per_iteration": per_it}


def dist_init(backend=None):
    """One process per GPU (or per CPU rank for gloo): env:// rendezvous."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600), **kw)
    return ws, rank, local


def replica_seed(base_seed: int, rank: int) -> int:
    """Replicas solve different seeded maps: rank r uses base_seed + r."""
    return base_seed + rank


def reduce_max(v: float, ws: int) -> float:
    """Maximum over ranks (the job's time is its slowest replica)."""
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference(args):
    ws, rank, _ = (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0)
    if rank != 0:
        return 0
    mesh, br0, opt, seed = build_case(args.workload)
    # The reference's CPU path (oracle restatement) needs about as many
    # iterations as the FP64 GPU path; the count of the seeded workload at
    # this size is recorded once per run by a short GPU-free estimate: the
    # projection uses the iteration count of the FP64 solve of this workload.
    ncg = args.ref_iterations or SOLVE_ITERATIONS.get((args.workload, args.ifprec), 0)
    if ncg <= 0:
        raise SystemExit(f"no iteration count known for {args.workload} with ifprec {args.ifprec}: "
                         "give --ref-iterations")
    vals = []
    for _ in range(args.warmup + args.steps):
        cb = cpu_baseline(mesh, br0, opt, args.ifprec, ncg, args.cpu_sample_iters)
        vals.append(cb["value"])
    v = float(np.mean(vals[args.warmup:]))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "ifprec": args.ifprec, "epscg": 1e-9, "seed": seed,
                       "parallelism": "replicas"},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pfss_255x361x721")
    ap.add_argument("--ifprec", type=int, default=2)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32_refined"])
    ap.add_argument("--epscg", type=float, default=1e-9)
    ap.add_argument("--cpu-sample-iters", type=int, default=0,
                    help="PCG iterations of the CPU sample (0: 20 with the diagonal preconditioner, 6 with ILU(0), "
                         "whose sequential sweeps take seconds per iteration)")
    ap.add_argument("--ref-iterations", type=int, default=0,
                    help="iteration count used to project the CPU sample (0: take it from a GPU solve)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--warm-start", default="auto",
                    help="FNO weights (.npz) for the learned initial guess; 'auto' uses "
                         "pot3d_b200/weights/fno_<workload>.npz when present; 'off' solves from zero")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain FP64 PCG (ifprec=1) solve timed beside the headline solve")
    ap.add_argument("--kernel-timing-only", action="store_true",
                    help="time the hot kernels briefly (stencil and update, or with --ifprec 2 the two "
                         "ILU(0) sweeps; used for ncu captures) and exit")
    args = ap.parse_args()
    if args.cpu_sample_iters <= 0:
        args.cpu_sample_iters = 6 if args.ifprec == 2 else 20

    if args.impl == "reference":
        return run_reference(args)

    ws, rank, local = dist_init()
    import torch
    from pot3d_b200.solver import Pot3dSolver

    torch.cuda.set_device(local)
    mesh, br0, opt, seed = build_case(args.workload, rank)
    s = Pot3dSolver(mesh, br0, option=opt, ifprec=args.ifprec, precision=args.precision, device=local)
    if args.kernel_timing_only:
        if args.ifprec == 2:
            fms, bms = s.time_sweeps(2)
            out = {}
            for name, t in (("k_dilu_wave<fwd>", fms), ("k_dilu_wave<bwd>", bms)):
                by = SWEEP_BYTES_PER_UNKNOWN[name] * s.N
                out[name] = {"ms": t, "gbs": by / (t * 1e-3) / 1e9}
            print(json.dumps({"workload": args.workload, "kernels": out}))
        else:
            ms, by = s.time_kernels(4)
            print(json.dumps({"workload": args.workload, "ms": list(ms), "gbs": list(by / (ms * 1e-3) / 1e9)}))
        s.close()
        return 0
    b = s.rhs()
    N = s.N
    xt = torch.zeros(N, dtype=torch.float64, device="cuda")
    rt = torch.empty(N, dtype=torch.float64, device="cuda")
    bt = torch.tensor(b, device="cuda")

    # Learned initial guess (FNO trained on this grid), inference timed as part of the solve.
    wpath = args.warm_start
    if wpath == "auto":
        cand = os.path.join(ROOT, "pot3d_b200", "weights", f"fno_{args.workload}.npz")
        wpath = cand if os.path.exists(cand) else "off"
    model = None
    if wpath != "off":
        from pot3d_b200.fno import FNO, grid_from_mesh
        from pot3d_b200.tc import LAUNCHES, check_errors
        from pot3d_b200.warmstart import Inputs
        model = FNO.load(wpath, grid_from_mesh(mesh))
        inputs = Inputs(model)
        v, sig = inputs.normalized(br0)
        br0n_h = torch.from_numpy(v).view(1, -1).pin_memory()
        br0n_d = br0n_h.cuda()
        sig_d = torch.tensor([sig], dtype=torch.float64, device="cuda")
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def guess_into(x):
        """Inference into x; returns (seconds, kernel launches)."""
        n0 = LAUNCHES[0]
        ev0.record()
        model.predict(inputs.build(br0n_d), sig_d, out=x.view(1, -1))
        ev1.record()
        ev1.synchronize()
        return ev0.elapsed_time(ev1) * 1e-3, LAUNCHES[0] - n0

    def solve_resident(learned=True):
        t_inf, n_inf = 0.0, 0
        if model is not None and learned:
            t_inf, n_inf = guess_into(xt)
        else:
            xt.zero_()
        rt.copy_(bt)
        torch.cuda.synchronize()
        ierr = s.cgsolve_dev(xt, rt, epscg=args.epscg)
        inf = s.last_info
        return ierr, inf.seconds + t_inf, inf.ncg, inf.epsn, inf.true_resid, inf.kernel_launches + n_inf, inf.n_refine

    for _ in range(args.warmup):
        solve_resident()
    barrier(ws)
    torch.cuda.synchronize()
    dev_times, ncgs, launches = [], [], 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            ierr, sec, ncg, epsn, tres, nl, nref = solve_resident()
            if ierr != 0:
                raise SystemExit(f"solve did not converge (ierr={ierr})")
            dev_times.append(sec)
            ncgs.append(ncg)
            launches += nl
    torch.cuda.synchronize()
    barrier(ws)
    t_dev = reduce_max(float(np.mean(dev_times)), ws)

    # End to end through the host-pointer C-ABI (H2D + solve + D2H) on pinned
    # host buffers; with the learned guess also the map's upload and the
    # guess's download.
    x_pin = torch.zeros(N, dtype=torch.float64, pin_memory=True)
    r_pin = torch.empty(N, dtype=torch.float64, pin_memory=True)
    x_h, r_h = x_pin.numpy(), r_pin.numpy()
    e2e = []
    h2d, d2h = 16 * N, 16 * N
    for it in range(args.steps):
        r_h[:] = b
        barrier(ws)
        t0 = time.perf_counter()
        if model is not None:
            br0n_d.copy_(br0n_h)
            guess_into(xt)
            x_pin.copy_(xt)
        else:
            x_h[:] = 0.0
        s.cgsolve(x_h, r_h, epscg=args.epscg)
        e2e.append(time.perf_counter() - t0)
    if model is not None:
        h2d += 4 * br0n_h.numel()
        d2h += 8 * N
        check_errors()
    t_e2e = reduce_max(float(np.mean(e2e)), ws)

    # The same solver from a zero guess (what the learned guess saves).
    zero_guess = None
    if model is not None:
        ierr0, sec0, ncg0, *_ = solve_resident(learned=False)
        zero_guess = {"seconds": reduce_max(sec0, ws), "iterations": ncg0}

    # Live kernel timing (CUDA events on the library's stream).
    kern = None
    if args.precision == "fp64" and args.ifprec != 2:
        ms, by = s.time_kernels(20)
        kern = {"k_stencil": {"ms": ms[0], "bytes": by[0], "gbs": by[0] / (ms[0] * 1e-3) / 1e9},
                "k_update": {"ms": ms[1], "bytes": by[1], "gbs": by[1] / (ms[1] * 1e-3) / 1e9}}
    elif args.ifprec == 2:
        fms, bms = s.time_sweeps(10)
        kern = {}
        for name, t in (("k_dilu_wave<fwd>", fms), ("k_dilu_wave<bwd>", bms)):
            by = SWEEP_BYTES_PER_UNKNOWN[name] * N
            kern[name] = {"ms": t, "bytes": by, "gbs": by / (t * 1e-3) / 1e9}

    # The plain FP64 PCG (diagonal preconditioner) on the same inputs.
    plain = None
    if args.ifprec == 2 and not args.no_plain:
        sp = Pot3dSolver(mesh, br0, option=opt, ifprec=1, precision="fp64", device=local)
        pt = []
        for it in range(2 if args.warmup > 0 else 1):
            xt.zero_()
            rt.copy_(bt)
            torch.cuda.synchronize()
            if sp.cgsolve_dev(xt, rt, epscg=args.epscg) != 0:
                raise SystemExit("plain FP64 solve did not converge")
            pt.append(sp.last_info.seconds)
        p_ncg = sp.last_info.ncg
        sp.close()
        t_plain = reduce_max(pt[-1], ws)
        plain = {"seconds": t_plain, "iterations": p_ncg, "ifprec": 1, "precision": "fp64",
                 "speedup": t_plain / t_dev}

    if rank != 0:
        s.close()
        return 0
    peak, psrc = peak_hbm()
    ncg = int(np.median(ncgs))
    bytes_per_iter = BYTES_PER_UNKNOWN_ITER[2 if args.ifprec == 2 else 1] * N
    overall_gbs = bytes_per_iter * ncg / t_dev / 1e9
    roofline = None
    if kern:
        dom = max(kern, key=lambda k: kern[k]["ms"])
        tr = measured_traffic(dom, args.workload)
        roofline = {"bound": "hbm", "kernel": dom, "achieved": kern[dom]["gbs"], "peak": peak, "unit": "GB/s",
                    "frac": kern[dom]["gbs"] / peak, "traffic": tr, "peak_source": f"{psrc} (MEASURED_PEAKS.json hbm_gbs)"
                    if psrc == "measured" else psrc,
                    "algorithmic_bytes_per_launch": kern[dom]["bytes"], "kernels": kern,
                    "solve_achieved_gbs": overall_gbs, "solve_frac": overall_gbs / peak}
    cb = None
    if not args.no_cpu_baseline and ws == 1:
        cb = cpu_baseline(mesh, br0, opt, args.ifprec, ncg, args.cpu_sample_iters)
        cb.pop("seconds_per_iteration", None)
    line = {
        "metric": METRIC, "value": t_dev, "unit": "s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_dev * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic",
        "config": {"workload": args.workload, "unknowns": N, "ifprec": args.ifprec, "precision": args.precision,
                   "initial_guess": "learned (FNO)" if model is not None else "zero",
                   "epscg": args.epscg, "seed": seed, "iterations": ncg, "parallelism": "replicas",
                   "l2": f"working set ~{(52 if args.ifprec != 2 else 104) * N / 1e9:.1f} GB >> 126 MB L2, no flush"},
        "e2e": {"value": t_e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": roofline, "cpu_baseline": cb, "clocks": clk.summary(),
        "gpu_launches": launches, "true_residual": tres, "epsn": epsn, "plain_fp64": plain,
        "warm_start": None if model is None else {"weights": os.path.relpath(wpath, ROOT), "zero_guess": zero_guess},
        "throughput_solves_per_s": ws / t_dev,
    }
    print(json.dumps(line), flush=True)
    s.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
