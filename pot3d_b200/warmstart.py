"""Learned warm start: training pairs from the solver, training, and the
held-out evaluation of the solve from the predicted guess against the solve
from zero.

    python -m pot3d_b200.warmstart --nr 127 --nt 181 --np 361 \\
        --train 2000 --test 200 --epochs 20 --out record.json [--save model.npz]
        [--ifprec 2] [--precision fp32_refined] [--plain]

Training pairs are (Br0 map, phi) of seeded synthetic PFSS cases solved by
the GPU solver (ILU(0), FP32-refined by default) to `--train-eps` (default
1e-9).  The evaluation solves every held-out case to the unchanged
tolerance (epscg 1e-9) from x = 0 and from the network's guess with the same
solver (and, with --plain, the plain FP64 diagonal PCG from zero); PCG
decides convergence either way, so a poor guess costs iterations, never
accuracy.  Each row records both iteration counts and times (inference
included) and how far the guessed solve's solution lies from the one from
zero.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import _lib, host
from .fno import FNO, _L, _stream, grid_from_mesh, new
from .solver import Pot3dSolver


def _set_br0(solver: Pot3dSolver, br0):
    L = _lib.lib()
    L.pot3d_gpu_set_br0.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    b = np.asfortranarray(br0, dtype=np.float64)
    _lib.check(L.pot3d_gpu_set_br0(solver._h, _lib.dptr(b)))


class Inputs:
    """Device-side assembly of the network inputs of a batch."""

    def __init__(self, model: FNO):
        import torch
        g = model.g
        self.model = model
        self.npos = g.nph * g.nth
        c = np.zeros((g.nph, g.nth, 3), np.float32)
        c[:, :, 0] = np.cos(g.th)[None, :]
        c[:, :, 1] = np.sin(g.th)[None, :]
        c[:, :, 2] = 1.0
        self.consts = torch.tensor(c.reshape(-1, 3)).cuda().contiguous()

    def normalized(self, br0):
        inner = np.asarray(br0)[1:-1, 1:-1]
        s = float(np.sqrt(np.mean(inner ** 2))) or 1.0
        return (inner / s).T.astype(np.float32).ravel(), s  # positions (phi, theta)

    def build(self, br0n_dev):
        """br0n_dev: FP32 [B, npos] on the device -> BF16 [B, nph, nth, 64]."""
        B = br0n_dev.shape[0]
        g = self.model.g
        x = new((B, g.nph, g.nth, 64), "bf16")
        from .tc import LAUNCHES
        LAUNCHES[0] += 1
        _lib.check(_L().pot3d_fno_inputs(C.c_void_p(br0n_dev.data_ptr()), C.c_void_p(self.consts.data_ptr()), B,
                                         self.npos, C.c_void_p(x.data_ptr()), _stream()))
        return x


def case_br0(mesh, seed, lmax, nbip):
    tn, pn, fi = host.synthetic_br(seed, lmax, nbip, mesh.nt, mesh.np)
    return host.br0_from_map(mesh, tn, pn, fi)


def generate(mesh, solver, inputs: Inputs, seeds, lmax, nbip, eps):
    """Solve every seeded case; returns device tensors br0n [S, npos] (FP32)
    and targets phi/sigma [S, npos*R] (BF16), plus solve statistics."""
    import torch
    S = len(seeds)
    N = solver.N
    br0n = torch.empty((S, inputs.npos), dtype=torch.float32, device="cuda")
    tgt = torch.empty((S, N), dtype=torch.bfloat16, device="cuda")
    sig = np.zeros(S)
    its, secs = [], []
    x = torch.zeros(N, dtype=torch.float64, device="cuda")
    r = torch.empty(N, dtype=torch.float64, device="cuda")
    for q, sd in enumerate(seeds):
        br0 = case_br0(mesh, sd, lmax, nbip)
        _set_br0(solver, br0)
        b = solver.rhs()
        x.zero_()
        r.copy_(torch.from_numpy(b))
        torch.cuda.synchronize()
        if solver.cgsolve_dev(x, r, epscg=eps) != 0:
            raise RuntimeError(f"training solve {sd} did not converge")
        its.append(solver.last_info.ncg)
        secs.append(solver.last_info.seconds)
        v, s = inputs.normalized(br0)
        br0n[q].copy_(torch.from_numpy(v))
        tgt[q].copy_(x / s)
        sig[q] = s
    return br0n, tgt, sig, {"iterations_mean": float(np.mean(its)), "solve_s_mean": float(np.mean(secs))}


def augment(br0n, tgt, nph, nth, R, shift, flip):
    """Exact symmetries of a case on a uniform periodic phi mesh (and a theta
    mesh symmetric about the equator): rotating Br0 in phi rotates phi, and
    reflecting north-south reflects it.  br0n [B, nph*nth], tgt [B, nph*nth*R]."""
    import torch
    B = br0n.shape[0]
    x = br0n.view(B, nph, nth)
    t = tgt.view(B, nph, nth, R)
    if shift:
        x = torch.roll(x, shifts=shift, dims=1)
        t = torch.roll(t, shifts=shift, dims=1)
    if flip:
        x = torch.flip(x, dims=(2,))
        t = torch.flip(t, dims=(2,))
    return x.reshape(B, -1).contiguous(), t.reshape(B, -1).contiguous()


def symmetric_mesh(mesh):
    """True when phi is uniform (rotations are exact) and theta is symmetric."""
    dph = np.asarray(mesh.dph)[1:-1]
    th = np.asarray(mesh.th)[1:-1]
    return bool(np.allclose(dph, dph[0], rtol=1e-12) and np.allclose(th + th[::-1], np.pi, atol=1e-12))


def train(model: FNO, inputs: Inputs, br0n, tgt, epochs, batch, lr, seed=0, log=None, augment_data=True):
    import torch
    S = br0n.shape[0]
    g = model.g
    rng = np.random.default_rng(seed)
    hist = []
    steps = max(1, S // batch)
    total = epochs * steps
    step = 0
    for ep in range(epochs):
        perm = rng.permutation(S)
        ep_loss = []
        for st in range(steps):
            idx = torch.tensor(perm[st * batch:(st + 1) * batch], device="cuda")
            xb = br0n.index_select(0, idx)
            t = tgt.index_select(0, idx)
            if augment_data:
                xb, t = augment(xb, t, g.nph, g.nth, g.R, int(rng.integers(g.nph)), bool(rng.integers(2)))
            x = inputs.build(xb.contiguous())
            loss, grad = model.loss_and_grad(x, t.contiguous())
            grads = model.backward(grad)
            # cosine decay of the learning rate
            cur = lr * 0.5 * (1.0 + np.cos(np.pi * step / total))
            model.adam_step(grads, lr=float(cur))
            ep_loss.append(loss)
            step += 1
        mean = float(torch.cat(ep_loss).mean().item())
        hist.append(mean)
        if log:
            log(f"epoch {ep}: relative squared error {mean:.4e}")
    return hist


def evaluate(model: FNO, inputs: Inputs, mesh, solver, seeds, lmax, nbip, eps=1e-9, plain=None):
    """Per held-out case: the solver to eps from zero and from the predicted
    guess (and, with `plain`, that solver from zero as the baseline)."""
    import torch
    N = solver.N
    rows = []
    x = torch.empty(N, dtype=torch.float64, device="cuda")
    r = torch.empty(N, dtype=torch.float64, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for sd in seeds:
        br0 = case_br0(mesh, sd, lmax, nbip)
        _set_br0(solver, br0)
        b = torch.from_numpy(solver.rhs()).cuda()
        x.zero_()
        r.copy_(b)
        torch.cuda.synchronize()
        if solver.cgsolve_dev(x, r, epscg=eps) != 0:
            raise RuntimeError(f"held-out solve {sd} from zero did not converge")
        z = solver.last_info
        xs = x.clone()
        v, s = inputs.normalized(br0)
        br0n = torch.from_numpy(v).cuda().view(1, -1)
        e0.record()
        guess = model.predict(inputs.build(br0n), [s])[0]
        e1.record()
        torch.cuda.synchronize()
        t_inf = e0.elapsed_time(e1) * 1e-3
        err = float(torch.linalg.norm(guess - xs) / torch.linalg.norm(xs))
        x.copy_(guess)
        r.copy_(b)
        torch.cuda.synchronize()
        if solver.cgsolve_dev(x, r, epscg=eps) != 0:
            raise RuntimeError(f"held-out solve {sd} from the guess did not converge")
        w = solver.last_info
        row = dict(seed=int(sd), ncg_zero=z.ncg, s_zero=z.seconds, ncg_guess=w.ncg, s_guess=w.seconds,
                   s_inference=t_inf, guess_rel_err=err, epsn_guess=w.epsn,
                   sol_rel_diff=float(torch.linalg.norm(x - xs) / torch.linalg.norm(xs)))
        if plain is not None:
            _set_br0(plain, br0)
            x.zero_()
            r.copy_(b)
            torch.cuda.synchronize()
            if plain.cgsolve_dev(x, r, epscg=eps) != 0:
                raise RuntimeError(f"plain solve {sd} did not converge")
            row["ncg_plain"] = plain.last_info.ncg
            row["s_plain"] = plain.last_info.seconds
        rows.append(row)
    a = lambda k: np.array([q[k] for q in rows])
    summ = dict(cases=len(rows), ncg_zero_mean=float(a("ncg_zero").mean()), ncg_guess_mean=float(a("ncg_guess").mean()),
                ncg_zero_median=float(np.median(a("ncg_zero"))), ncg_guess_median=float(np.median(a("ncg_guess"))),
                s_zero_mean=float(a("s_zero").mean()),
                s_guess_mean=float((a("s_guess") + a("s_inference")).mean()),
                s_inference_mean=float(a("s_inference").mean()),
                guess_rel_err_mean=float(a("guess_rel_err").mean()),
                guess_rel_err_max=float(a("guess_rel_err").max()),
                sol_rel_diff_max=float(a("sol_rel_diff").max()),
                iteration_ratio=float(a("ncg_guess").mean() / a("ncg_zero").mean()),
                time_ratio=float((a("s_guess") + a("s_inference")).mean() / a("s_zero").mean()),
                fewer_iterations_cases=int((a("ncg_guess") < a("ncg_zero")).sum()))
    if plain is not None:
        summ["ncg_plain_mean"] = float(a("ncg_plain").mean())
        summ["s_plain_mean"] = float(a("s_plain").mean())
        summ["speedup_learned_vs_plain"] = summ["s_plain_mean"] / summ["s_guess_mean"]
    return summ, rows


def evaluate_saved(args, mesh):
    """The --evaluate record: a saved operator on this grid's held-out seeds."""
    import torch
    z = np.load(args.evaluate)
    model = FNO.load_resampled(args.evaluate, mesh)
    inputs = Inputs(model)
    solver = Pot3dSolver(mesh, case_br0(mesh, args.test_seed0, args.lmax, args.nbip), ifprec=args.ifprec,
                         precision=args.precision)
    plain = Pot3dSolver(mesh, case_br0(mesh, args.test_seed0, args.lmax, args.nbip), ifprec=1) if args.plain else None
    t0 = time.time()
    summ, rows = evaluate(model, inputs, mesh, solver, range(args.test_seed0, args.test_seed0 + args.test),
                          args.lmax, args.nbip, plain=plain)
    torch.cuda.synchronize()
    cfg = {k: v for k, v in vars(args).items() if k in ("nr", "nt", "np", "lmax", "nbip", "test", "test_seed0",
                                                       "ifprec", "precision", "plain", "evaluate")}
    cfg["trained_interior_theta_phi_r"] = "x".join(str(int(v)) for v in z["grid"][:3])
    cfg["radial_levels_resampled"] = getattr(model, "R_out", None) is not None
    rep = dict(config=cfg, evaluation=dict(seconds=time.time() - t0, **summ), cases=rows)
    with open(args.out, "w") as fh:
        json.dump(rep, fh, indent=1)
    print(json.dumps(summ), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nr", type=int, default=127)
    ap.add_argument("--nt", type=int, default=181)
    ap.add_argument("--np", type=int, default=361)
    ap.add_argument("--lmax", type=int, default=40)
    ap.add_argument("--nbip", type=int, default=20)
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--test", type=int, default=200)
    ap.add_argument("--train-seed0", type=int, default=1000)
    ap.add_argument("--test-seed0", type=int, default=5000)
    ap.add_argument("--train-eps", type=float, default=1e-9)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default="warmstart.json")
    ap.add_argument("--save", default="")
    ap.add_argument("--no-augment", action="store_true")
    ap.add_argument("--ifprec", type=int, default=2, help="preconditioner of the generating and evaluating solves")
    ap.add_argument("--precision", default="fp32_refined", choices=["fp64", "fp32_refined"])
    ap.add_argument("--plain", action="store_true", help="also time the plain FP64 diagonal PCG from zero")
    ap.add_argument("--evaluate", default="",
                    help="only evaluate the saved operator at this path on the held-out seeds of this grid (run on "
                         "the grid's theta-phi points, its radial levels interpolated when the grids differ)")
    args = ap.parse_args(argv)
    import torch
    mesh = host.make_mesh(args.nr, args.nt, args.np)
    if args.evaluate:
        return evaluate_saved(args, mesh)
    solver = Pot3dSolver(mesh, case_br0(mesh, args.train_seed0, args.lmax, args.nbip), ifprec=args.ifprec,
                         precision=args.precision)
    model = FNO(grid_from_mesh(mesh))
    inputs = Inputs(model)
    t0 = time.time()
    br0n, tgt, sig, gstat = generate(mesh, solver, inputs, range(args.train_seed0, args.train_seed0 + args.train),
                                     args.lmax, args.nbip, args.train_eps)
    t1 = time.time()
    print(f"generated {args.train} pairs in {t1 - t0:.1f} s ({gstat})", flush=True)
    torch.cuda.synchronize()
    aug = symmetric_mesh(mesh) and not args.no_augment
    hist = train(model, inputs, br0n, tgt, args.epochs, args.batch, args.lr, log=lambda s: print(s, flush=True),
                 augment_data=aug)
    torch.cuda.synchronize()
    t2 = time.time()
    from .tc import check_errors
    check_errors()
    del br0n, tgt
    plain = Pot3dSolver(mesh, case_br0(mesh, args.test_seed0, args.lmax, args.nbip), ifprec=1) if args.plain else None
    summ, rows = evaluate(model, inputs, mesh, solver, range(args.test_seed0, args.test_seed0 + args.test),
                          args.lmax, args.nbip, plain=plain)
    t3 = time.time()
    rep = dict(config=vars(args), generation=dict(seconds=t1 - t0, **gstat), training=dict(seconds=t2 - t1,
               loss_history=hist), evaluation=dict(seconds=t3 - t2, **summ), cases=rows)
    with open(args.out, "w") as fh:
        json.dump(rep, fh, indent=1)
    print(json.dumps(summ), flush=True)
    if args.save:
        model.save(args.save)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
