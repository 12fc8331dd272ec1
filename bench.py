"""Benchmark: seconds to solve POT3D's PCG to epsn <= 1e-9 on one B200.

One step = one complete solve of the PFSS workload 255x361x721 (65.3 M
unknowns, seeded synthetic Br: spherical harmonics l<=40 plus 20 bipoles)
to the reference's stopping rule epsn < epscg = 1e-9 (ernorm,
src/pot3d.F90:4430-4433), by the headline method: the learned initial
guess (the FNO trained on 2000 solves at 127x181x361, run on this grid's
theta-phi points with its radial levels interpolated onto this mesh, its
inference inside the timed region) followed by FP32-inner / FP64-refined PCG with the reference's
ILU(0) preconditioner (ifprec=2).  Timed in the same run, on the same
inputs: the plain FP64 PCG with the diagonal preconditioner (ifprec=1, the
reference's default) and FP64 PCG with ILU(0) from zero (same
preconditioner), both to 1e-9.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME] [--ifprec 1|2] [--precision fp64|fp32_refined]
                    [--warm-start auto|off|PATH] [--no-plain] [--no-parity]

value: device time of the solve (CUDA events on the library's stream around
the PCG initialisation and iterations, plus the guess's inference on
torch's stream), inputs resident in HBM.
e2e: the same solve end to end from page-locked host buffers, wall clock:
the upload of the map (the guess is inferred from it on the device) and of
the right-hand side, the solve through the C-ABI (pot3d_gpu_cgsolve_dev),
and the download of x and r (cgsolve's outputs).
The working set (about 3 GB of vectors plus 2.5 GB of sweep coefficient
streams) is 40x the 126 MB L2, so no flush is needed between steps.
parity: the headline method solved to 1e-11 against FP64 PCG (ILU(0)) to
1e-11 on the GPU and against the oracle's FP64 solve (tests/golden fixture):
phi relative L2 and energy relative errors.

The CPU legs (cpu_baseline and --impl reference) time the oracle -- the C
restatement of the reference's CPU PCG -- on the host cores, on a case the
oracle builds by itself (its mesh, the seeded map generator and readbr),
over a bounded sample of PCG iterations projected to the iteration count
of the oracle's own full solve of the workload (tests/golden fixture).

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
# Algorithmic DRAM bytes per unknown (matrix-free coefficients, each vector
# touched once per fused pass): FP64 PCG iteration 80 (ifprec=1) / 104
# (ifprec=2); FP32-inner iteration 40 / 64; each FP64 reliable update 24.
# The ILU(0) application moves 12 B forward (r32, d, y) and 12 B backward
# (y, d, z32).  In the refined mode's inner iteration the forward sweep also
# applies the residual half of the update (q32 read, r32 written: +8 B; its
# r32 read is the sweep's own) and the backward sweep forms rho = r.z (r32
# read: +4 B; z is its own output).
BYTES_PER_UNKNOWN_ITER = {("fp64", 1): 80.0, ("fp64", 2): 104.0, ("fp32_refined", 1): 40.0,
                          ("fp32_refined", 2): 64.0}
BYTES_PER_REFINE = 24.0
SWEEP_BYTES_PER_UNKNOWN = {"k_dilu_wave<fwd>": 12.0, "k_dilu_wave<bwd>": 12.0,
                           "k_dilu_wave<fwd,fused>": 20.0, "k_dilu_wave<bwd,fused>": 16.0}


def sweep_names(precision: str):
    """The sweep kernels a solver of this arithmetic iterates with (what
    pot3d_gpu_time_sweeps times)."""
    if precision == "fp32_refined":
        return ("k_dilu_wave<fwd,fused>", "k_dilu_wave<bwd,fused>")
    return ("k_dilu_wave<fwd>", "k_dilu_wave<bwd>")
FALLBACK_HBM_GBS = 6650.0
GOLDEN = os.path.join(ROOT, "tests", "golden")


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


def oracle_fixture(workload: str, ifprec: int):
    """The oracle's full solve of the workload (tests/golden), or None."""
    p = os.path.join(GOLDEN, f"{workload}_oracle_ifprec{ifprec}.json")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        rec = json.load(fh)
    z = np.load(p[:-5] + ".npz")
    rec["phi_slices"] = z["phi_slices"]
    rec["slice_i"] = z["slice_i"]
    rec["stride"] = int(z["stride"])
    return rec


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


def workload_params(name: str, rank: int = 0):
    from pot3d_b200 import host
    w = dict(host.WORKLOADS[name])
    opt = w.pop("option", "ss")
    dnb = w.pop("do_not_balance_flux", False)
    w["seed"] = replica_seed(w["seed"], rank)
    return w, opt, dnb


def build_case(name: str, rank: int = 0):
    from pot3d_b200 import host
    w, opt, dnb = workload_params(name, rank)
    mesh, br0 = host.pfss_case(w["nr"], w["nt"], w["np"], w["lmax"], w["nbip"], w["seed"], option=opt,
                               do_not_balance_flux=dnb)
    return mesh, br0, opt, w["seed"]


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


def oracle_case(name: str, seed: int, option: str, dnb: bool):
    """(mesh, br0) of the workload built by the oracle alone (no product
    library involved)."""
    O = _oracle()
    from pot3d_b200 import host  # workload table only (pure Python)
    w = host.WORKLOADS[name]
    return O.pfss_case(w["nr"], w["nt"], w["np"], w["lmax"], w["nbip"], seed, option=option,
                       do_not_balance_flux=dnb)


def cpu_reference_time(workload, ifprec, sample_iters, rank=0):
    """The oracle (CPU restatement of the reference's PCG, OpenMP on the
    host cores; the ILU(0) sweeps sequential as in lusol) on the workload:
    the full solve when it is small, otherwise `sample_iters` iterations
    projected to the iteration count of the oracle's full solve."""
    O = _oracle()
    w, opt, dnb = workload_params(workload, rank)
    t0 = time.perf_counter()
    mesh, br0 = oracle_case(workload, w["seed"], opt, dnb)
    s = O.Solver(mesh, br0, option=opt, ifprec=ifprec)
    b = s.rhs()
    t1 = time.perf_counter()
    N = s.N
    fix = oracle_fixture(workload, ifprec) if rank == 0 else None
    if N <= 2_000_000:  # small grids: the whole solve
        out = s.cgsolve(np.zeros(N), b, epscg=1e-9)
        t2 = time.perf_counter()
        rec = {"value": t2 - t1, "unit": "s", "cores": O.threads(), "kind": "port", "projected": False,
               "sample": f"oracle full PCG solve (ifprec={ifprec}) of {mesh.nr}x{mesh.nt}x{mesh.np} to 1e-9: "
                         f"{out['ncg']} iterations (set-up {t1 - t0:.1f} s not included)",
               "iterations": out["ncg"]}
    else:
        if fix is None or fix.get("iterations_to_1e-9") is None:
            raise SystemExit(f"no oracle solve of {workload} (ifprec {ifprec}) in tests/golden: run "
                             f"tests/golden/make_c2_oracle.py")
        ncg_full = int(fix["iterations_to_1e-9"])
        out = s.cgsolve(np.zeros(N), b, ncgmax=sample_iters, epscg=0.0)
        t2 = time.perf_counter()
        per_it = (t2 - t1) / max(1, out["ncg"])
        rec = {"value": per_it * ncg_full, "unit": "s", "cores": O.threads(), "kind": "port", "projected": True,
               "sample": f"oracle PCG (ifprec={ifprec}) on {mesh.nr}x{mesh.nt}x{mesh.np}: set-up, then "
                         f"{out['ncg']} iterations timed ({per_it * 1e3:.0f} ms each), projected to the "
                         f"{ncg_full} iterations of the oracle's own full solve to 1e-9 (tests/golden); "
                         f"set-up {t1 - t0:.1f} s not included",
               "iterations": ncg_full, "seconds_per_iteration": per_it}
    del s
    return rec


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
    """The reference's CPU PCG (the oracle) on the same workload: rank 0
    only; one bounded sample, projected (see cpu_reference_time)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cb = cpu_reference_time(args.workload, args.ifprec, args.ref_sample_iters)
    v = cb["value"]
    w, opt, _ = workload_params(args.workload)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "ifprec": args.ifprec, "epscg": args.epscg, "seed": w["seed"],
                       "option": opt, "parallelism": "replicas",
                       "method": "the reference's CPU cgsolve from zero (FP64, ILU(0) sweeps sequential)"},
            "projected": cb["projected"], "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_legacy_lu(args):
    """The legacy external-LU symbols (the -DCUSPARSE Fortran host's path,
    src/lusol_cusparse.c:64,309,374) on the workload's diacsr CSR (built by
    the oracle): wall time of load (factorisation) and of one application,
    as the Fortran host sees them, and the application checked bit for bit
    against the oracle's lusol.  The reference's own cuSPARSE shim is not
    run (it crashed in this process: see the reason in the output)."""
    import ctypes as C

    import torch
    O = _oracle()
    w, opt, dnb = workload_params(args.workload)
    mesh, br0 = oracle_case(args.workload, w["seed"], opt, dnb)
    o = O.Solver(mesh, br0, option=opt, ifprec=1)
    ia, ja, a = o.csr()
    N = o.N
    del o
    rhs = np.random.default_rng(0).standard_normal(N)
    out = {"workload": args.workload, "N": N, "nnz": int(ia[-1] - 1)}
    z = {}
    libs = {"ours": os.path.join(ROOT, "pot3d_b200", "libpot3d_gpu.so")}
    out["reference_cusparse"] = {
        "unavailable": "the reference's src/lusol_cusparse.c, built against the image's cuSPARSE and driven with "
                       "this CSR from a torch process, crashed the process (SIGSEGV in load_external_lu_solver); "
                       "not run again"}
    for name, path in libs.items():
        L = C.CDLL(path)  # RTLD_LOCAL: each library's symbols resolve on its own handle
        L.load_external_lu_solver.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.external_lu_solver.argtypes = [C.c_void_p]
        ia_d = torch.tensor(ia, dtype=torch.int32, device="cuda")
        ja_d = torch.tensor(ja, dtype=torch.int32, device="cuda")
        a_d = torch.tensor(a, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.load_external_lu_solver(a_d.data_ptr(), ia_d.data_ptr(), ja_d.data_ptr(), N, int(ia[-1]))
        torch.cuda.synchronize()
        t_load = time.perf_counter() - t0
        x = torch.tensor(rhs, device="cuda")
        L.external_lu_solver(x.data_ptr())
        torch.cuda.synchronize()
        z[name] = x.cpu().numpy()
        ts = []
        for _ in range(args.warmup + args.steps):
            x.copy_(torch.tensor(rhs, device="cuda"))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            L.external_lu_solver(x.data_ptr())
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        L.unload_external_lu_solver()
        out[name] = {"load_s": t_load, "apply_ms": 1e3 * float(np.mean(ts[args.warmup:])),
                     "apply_ms_min": 1e3 * float(np.min(ts[args.warmup:]))}
        del ia_d, ja_d, a_d, x
    if N <= 2_000_000:  # the oracle's lusol on the host: bit for bit
        o = O.Solver(mesh, br0, option=opt, ifprec=2)
        out["ours"]["bitwise_vs_oracle_lusol"] = bool(np.array_equal(z["ours"], o.prec(rhs)))
        del o
    print(json.dumps({"legacy_lu": out}), flush=True)
    return 0


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pfss_255x361x721")
    ap.add_argument("--ifprec", type=int, default=2)
    ap.add_argument("--precision", default="fp32_refined", choices=["fp64", "fp32_refined"])
    ap.add_argument("--epscg", type=float, default=1e-9)
    ap.add_argument("--cpu-sample-iters", type=int, default=0,
                    help="oracle PCG iterations of the CPU baseline sample (0: 10 with ILU(0), whose sequential "
                         "sweeps take seconds per iteration, 60 with the diagonal preconditioner)")
    ap.add_argument("--ref-sample-iters", type=int, default=30,
                    help="oracle PCG iterations of the reference arm's sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--warm-start", default="auto",
                    help="FNO weights (.npz) for the learned initial guess, run on the workload's grid; "
                         "'auto' uses pot3d_b200/weights/fno_<workload>.npz when present, else the operator "
                         "trained at 127x181x361; 'off' solves from zero")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the FP64 solves timed beside the headline solve")
    ap.add_argument("--no-parity", action="store_true", help="skip the 1e-11 parity solves")
    ap.add_argument("--legacy-lu", action="store_true",
                    help="time the legacy external-LU symbols against the reference's cuSPARSE shim and exit")
    ap.add_argument("--kernel-timing-only", action="store_true",
                    help="time the hot kernels briefly (stencil and update, or with --ifprec 2 the two "
                         "ILU(0) sweeps; used for ncu captures) and exit")
    args = ap.parse_args()
    if args.cpu_sample_iters <= 0:
        args.cpu_sample_iters = 10 if args.ifprec == 2 else 60

    if args.impl == "reference":
        return run_reference(args)
    if args.legacy_lu:
        return run_legacy_lu(args)

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
            for name, t in zip(sweep_names(args.precision), (fms, bms)):
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

    # Learned initial guess, inference timed as part of the solve: the FNO
    # trained for this grid when there is one, else the operator trained at
    # 127x181x361 run on this grid (resolution-free in theta-phi, its radial
    # levels interpolated onto this mesh's).  Trained on PFSS maps, it also
    # starts the open-field workload closer than zero (fewer iterations to
    # the same tolerance), though far from its solution.
    wpath = args.warm_start
    if wpath == "auto":
        cand = os.path.join(ROOT, "pot3d_b200", "weights", f"fno_{args.workload}.npz")
        base = os.path.join(ROOT, "pot3d_b200", "weights", "fno_pfss_127x181x361.npz")
        wpath = cand if os.path.exists(cand) else base
    model = None
    if wpath != "off":
        from pot3d_b200.fno import FNO
        from pot3d_b200.tc import LAUNCHES, check_errors
        from pot3d_b200.warmstart import Inputs
        model = FNO.load_resampled(wpath, mesh)
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

    def solve_resident(solver=s, learned=True, epscg=args.epscg):
        t_inf, n_inf = 0.0, 0
        if model is not None and learned:
            t_inf, n_inf = guess_into(xt)
        else:
            xt.zero_()
        rt.copy_(bt)
        torch.cuda.synchronize()
        ierr = solver.cgsolve_dev(xt, rt, epscg=epscg)
        inf = solver.last_info
        return dict(ierr=ierr, seconds=inf.seconds + t_inf, ncg=inf.ncg, epsn=inf.epsn, true_resid=inf.true_resid,
                    launches=inf.kernel_launches + n_inf, n_refine=inf.n_refine, inference_s=t_inf)

    for _ in range(args.warmup):
        solve_resident()
    barrier(ws)
    torch.cuda.synchronize()
    steps = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            st = solve_resident()
            if st["ierr"] != 0:
                raise SystemExit(f"solve did not converge (ierr={st['ierr']})")
            steps.append(st)
    torch.cuda.synchronize()
    barrier(ws)
    t_dev = reduce_max(float(np.mean([q["seconds"] for q in steps])), ws)
    x_timed = xt.cpu().numpy()
    fallback = s.refine_info()[1] if args.precision == "fp32_refined" else 0

    # End to end, wall clock, from page-locked host buffers: the inputs (the
    # right-hand side, and the boundary map the guess is inferred from) go up,
    # the result (x and the residual r, cgsolve's outputs) comes down.  From
    # zero: the host-pointer C-ABI (pot3d_gpu_cgsolve: x and r uploaded, x
    # and r downloaded).  With the learned guess: the map's upload, the
    # inference into the device x, r's upload, the device-pointer C-ABI
    # (pot3d_gpu_cgsolve_dev) and the downloads of x and r.
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
            rt.copy_(r_pin)
            if s.cgsolve_dev(xt, rt, epscg=args.epscg) != 0:
                raise SystemExit("e2e solve did not converge")
            x_pin.copy_(xt)
            r_pin.copy_(rt)
            torch.cuda.synchronize()
        else:
            x_h[:] = 0.0
            if s.cgsolve(x_h, r_h, epscg=args.epscg) != 0:
                raise SystemExit("e2e solve did not converge")
        e2e.append(time.perf_counter() - t0)
    if model is not None:
        h2d = 8 * N + 4 * br0n_h.numel()
        check_errors()
    t_e2e = reduce_max(float(np.mean(e2e)), ws)

    # The same method from a zero guess (what the learned guess saves).
    zero_guess = None
    if model is not None:
        z0 = solve_resident(learned=False)
        zero_guess = {"seconds": reduce_max(z0["seconds"], ws), "iterations": z0["ncg"]}

    # Live kernel timing (CUDA events on the library's stream).
    kern = None
    if args.ifprec == 2:
        fms, bms = s.time_sweeps(10)
        kern = {}
        for name, t in zip(sweep_names(args.precision), (fms, bms)):
            by = SWEEP_BYTES_PER_UNKNOWN[name] * N
            kern[name] = {"ms": t, "bytes": by, "gbs": by / (t * 1e-3) / 1e9}
    elif args.precision == "fp64":
        ms, by = s.time_kernels(20)
        kern = {"k_stencil": {"ms": ms[0], "bytes": by[0], "gbs": by[0] / (ms[0] * 1e-3) / 1e9},
                "k_update": {"ms": ms[1], "bytes": by[1], "gbs": by[1] / (ms[1] * 1e-3) / 1e9}}

    # FP64 PCG beside it: ILU(0) from zero (same preconditioner) and the
    # diagonal preconditioner (the reference's default), same inputs.  One
    # FP64 solver at a time besides the headline one (the largest workload
    # needs ~70 GB per solver).
    plain = same_prec = parity = None
    if not args.no_plain or not args.no_parity:
        s64 = Pot3dSolver(mesh, br0, option=opt, ifprec=2, precision="fp64", device=local)
        if not args.no_plain:
            r64 = [solve_resident(s64, learned=False) for _ in range(2 if args.warmup > 0 else 1)]
            if any(q["ierr"] for q in r64):
                raise SystemExit("the FP64 ILU(0) solve did not converge")
            t64 = reduce_max(r64[-1]["seconds"], ws)
            same_prec = {"seconds": t64, "iterations": r64[-1]["ncg"], "ifprec": 2, "precision": "fp64",
                         "initial_guess": "zero", "speedup": t64 / t_dev}
        if not args.no_parity:
            # Parity: the headline method and FP64 PCG both to 1e-11; the timed
            # 1e-9 solution against the FP64 1e-11 one; against the oracle's.
            def fields(x):
                out = s.fields(x, want=("phi", "w"))
                return out["phi"], out["w"]
            ref = solve_resident(s64, learned=False, epscg=1e-11)
            x64 = xt.cpu().numpy()
            mine = solve_resident(s, learned=True, epscg=1e-11)
            x11 = xt.cpu().numpy()
            phi64, w64 = fields(x64)
            del x64
            phi11, w11 = fields(x11)
            del x11
            parity = {"epscg": 1e-11, "fp64_ilu_iterations": ref["ncg"], "method_iterations": mine["ncg"],
                      "phi_rel_l2": rel_l2(phi11, phi64),
                      "energy_rel_err": float(np.max(np.abs(w11 - w64) / np.abs(w64)))}
            phi9, w9 = fields(x_timed)
            parity["timed_1e-9_phi_rel_l2"] = rel_l2(phi9, phi64)
            parity["timed_1e-9_energy_rel_err"] = float(np.max(np.abs(w9 - w64) / np.abs(w64)))
            parity["energies_1e-11"] = w11.tolist()
            del phi9, phi64
            parity["oracle"] = {}
            for pf in (2, 1):
                fix = oracle_fixture(args.workload, pf) if rank == 0 else None
                if fix is None:
                    continue
                wo = np.asarray(fix["energy"])
                sl = np.stack([phi11[i - 1, ::fix["stride"], ::fix["stride"]] for i in fix["slice_i"]])
                parity["oracle"][f"ifprec{pf}"] = {
                    "source": f"tests/golden/{args.workload}_oracle_ifprec{pf} (oracle FP64 PCG to 1e-11, "
                              f"{fix['iterations']} iterations)",
                    "energy_rel_err": float(np.max(np.abs(w11 - wo) / np.abs(wo))),
                    "phi_slices_rel_l2": rel_l2(sl, fix["phi_slices"])}
            del phi11
        s64.close()
    if not args.no_plain:
        sp = Pot3dSolver(mesh, br0, option=opt, ifprec=1, precision="fp64", device=local)
        pt = [solve_resident(sp, learned=False) for _ in range(2 if args.warmup > 0 else 1)]
        sp.close()
        if any(q["ierr"] for q in pt):
            raise SystemExit("the plain FP64 solve did not converge")
        t_plain = reduce_max(pt[-1]["seconds"], ws)
        plain = {"seconds": t_plain, "iterations": pt[-1]["ncg"], "ifprec": 1, "precision": "fp64",
                 "initial_guess": "zero", "speedup": t_plain / t_dev,
                 "achieved_gbs": 80.0 * N * pt[-1]["ncg"] / t_plain / 1e9}

    if rank != 0:
        s.close()
        return 0
    peak, psrc = peak_hbm()
    ncg = int(np.median([q["ncg"] for q in steps]))
    nref = int(np.median([q["n_refine"] for q in steps]))
    algo_bytes = BYTES_PER_UNKNOWN_ITER[(args.precision, 2 if args.ifprec == 2 else 1)] * N * ncg + \
        BYTES_PER_REFINE * N * nref
    overall_gbs = algo_bytes / t_dev / 1e9
    roofline = None
    if kern:
        dom = max(kern, key=lambda k: kern[k]["ms"])
        tr = measured_traffic(dom, args.workload)
        roofline = {"bound": "hbm", "kernel": dom, "achieved": kern[dom]["gbs"], "peak": peak, "unit": "GB/s",
                    "frac": kern[dom]["gbs"] / peak, "traffic": tr,
                    "peak_source": f"{psrc} (MEASURED_PEAKS.json hbm_gbs)" if psrc == "measured" else psrc,
                    "algorithmic_bytes_per_launch": kern[dom]["bytes"], "kernels": kern,
                    "solve_algorithmic_bytes": algo_bytes, "solve_achieved_gbs": overall_gbs,
                    "solve_frac": overall_gbs / peak}
    cb = None
    if not args.no_cpu_baseline and ws == 1:
        cb = cpu_reference_time(args.workload, args.ifprec, args.cpu_sample_iters)
        cb.pop("seconds_per_iteration", None)
    line = {
        "metric": METRIC, "value": t_dev, "unit": "s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_dev * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic",
        "config": {"workload": args.workload, "unknowns": N, "ifprec": args.ifprec, "precision": args.precision,
                   "initial_guess": "learned (FNO)" if model is not None else "zero",
                   "epscg": args.epscg, "seed": seed, "iterations": ncg, "reliable_updates": nref,
                   "fp64_fallback_iterations": fallback, "parallelism": "replicas",
                   "l2": f"working set ~{(40 if args.ifprec != 2 else 84) * N / 1e9:.1f} GB >> 126 MB L2, no flush"},
        "e2e": {"value": t_e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": roofline, "cpu_baseline": cb, "clocks": clk.summary(),
        "gpu_launches": int(np.sum([q["launches"] for q in steps])), "true_residual": steps[-1]["true_resid"],
        "epsn": steps[-1]["epsn"], "inference_s": steps[-1]["inference_s"],
        "plain_fp64": plain, "fp64_same_preconditioner": same_prec, "parity": parity,
        "warm_start": None if model is None else {
            "weights": os.path.relpath(wpath, ROOT),
            "trained_interior_theta_phi_r": "x".join(str(int(v)) for v in np.load(wpath)["grid"][:3]),
            "radial_levels_resampled": getattr(model, "R_out", None) is not None, "zero_guess": zero_guess},
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
