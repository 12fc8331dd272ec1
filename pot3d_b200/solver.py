"""Python mirror of POT3D's solve interface over the C-ABI.

``Pot3dSolver`` holds one set-up solve (potfld's matrix and preconditioner
load, src/pot3d.F90:3907-3935) on the GPU; ``cgsolve`` keeps the reference
contract of cgsolve(x, r, N, ierr) (src/pot3d.F90:4231-4369): x is the
guess on entry and the solution on exit, r the RHS on entry and the residual
on exit, and ierr is 0 when converged and 1 when ncgmax was exceeded.
``potfld`` runs the whole reference sequence: RHS by the boundary trick,
PCG, phi with ghosts, and the magnetic energies of magnetic_energy.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import SolveInfo, check, dptr, fptr
from .host import PM_R1, Mesh

PRECISION = {"fp64": 0, "fp32_refined": 1}


class Pot3dSolver:
    def __init__(self, mesh: Mesh, br0, option: str = "ss", ifprec: int = 1, precision: str = "fp64",
                 br1=None, device: int = -1):
        self.mesh = mesh
        self.option = option
        self.ifprec = ifprec
        self.precision = precision
        self._br0 = np.asfortranarray(br0, dtype=np.float64)
        self._br1 = None if br1 is None else np.asfortranarray(br1, dtype=np.float64)
        self._mc = mesh.cstruct()
        h = C.c_void_p()
        check(_lib.lib().pot3d_gpu_create(C.byref(self._mc), dptr(self._br0),
                                          None if self._br1 is None else dptr(self._br1), PM_R1[option], ifprec,
                                          PRECISION[precision], device, C.byref(h)))
        self._h = h
        self.N = int(_lib.lib().pot3d_gpu_size(h))
        self.last_info = None

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().pot3d_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- reference-shaped API ------------------------------------------
    def set_br0(self, br0):
        """Replace the boundary map (nt, np), keeping mesh, operator and
        preconditioner (set_flux for a new map)."""
        b = np.asfortranarray(br0, dtype=np.float64)
        if b.shape != (self.mesh.nt, self.mesh.np):
            raise ValueError("br0 must have shape (nt, np)")
        self._br0 = b
        check(_lib.lib().pot3d_gpu_set_br0(self._h, dptr(b)))

    def br0_from_map(self, tn, pn, fi, option=None, do_not_balance_flux=False) -> np.ndarray:
        """readbr on the device: interpolate the map fi[ntn, npn] (Fortran
        axis order, scales tn, pn) onto the mesh, pole rows, flux balance and
        'open' |Br|; the result becomes this solve's br0 and is returned
        (nt, np) in Fortran order."""
        from .host import OPTION_CODE
        opt = self.option if option is None else option
        fi = np.asfortranarray(np.asarray(fi, dtype=np.float64))
        tn = np.ascontiguousarray(tn, dtype=np.float64)
        pn = np.ascontiguousarray(pn, dtype=np.float64)
        out = np.zeros((self.mesh.nt, self.mesh.np), order="F")
        check(_lib.lib().pot3d_gpu_br0_from_map(self._h, fi.shape[0], fi.shape[1], dptr(tn), dptr(pn), dptr(fi),
                                                OPTION_CODE[opt], int(do_not_balance_flux), dptr(out)))
        self._br0 = out
        return out

    def rhs(self) -> np.ndarray:
        b = np.zeros(self.N)
        check(_lib.lib().pot3d_gpu_rhs(self._h, dptr(b)))
        return b

    def cgsolve(self, x: np.ndarray, r: np.ndarray, ncgmax: int = 10_000_000, epscg: float = 1e-9) -> int:
        """In place on host arrays x (guess -> solution), r (RHS -> residual)."""
        for a in (x, r):
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.size != self.N:
                raise ValueError("x and r must be contiguous float64 arrays of length N")
        ierr = C.c_int(1)
        info = SolveInfo()
        check(_lib.lib().pot3d_gpu_cgsolve(self._h, dptr(x), dptr(r), self.N, ncgmax, epscg, C.byref(ierr),
                                           C.byref(info)))
        self.last_info = info
        return ierr.value

    def cgsolve_dev(self, x, r, ncgmax: int = 10_000_000, epscg: float = 1e-9) -> int:
        """Same on CUDA tensors (device pointers), as the Fortran host's
        use_device_addr arrays."""
        for a in (x, r):
            if not a.is_cuda or a.dtype.itemsize != 8 or not a.is_contiguous() or a.numel() != self.N:
                raise ValueError("x and r must be contiguous float64 CUDA tensors of length N")
        ierr = C.c_int(1)
        info = SolveInfo()
        check(_lib.lib().pot3d_gpu_cgsolve_dev(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(r.data_ptr()),
                                               self.N, ncgmax, epscg, C.byref(ierr), C.byref(info)))
        self.last_info = info
        return ierr.value

    def set_refine(self, refine_ratio: float = 1e-4, stall_drop: float = 0.5, stall_limit: int = 2):
        """Reliable-update and stagnation controls of the FP32-refined solve."""
        check(_lib.lib().pot3d_gpu_set_refine(self._h, refine_ratio, stall_drop, stall_limit))

    def refine_info(self):
        """(reliable updates, FP64 iterations after a switch to FP64 PCG) of
        the last refined solve."""
        nr, fb = C.c_int(0), C.c_int(0)
        check(_lib.lib().pot3d_gpu_refine_info(self._h, C.byref(nr), C.byref(fb)))
        return nr.value, fb.value

    def test_sweep_stall(self, spin_limit: int = 1 << 12) -> int:
        """Status code of an ILU(0) forward sweep run with one tile left
        undone (POT3D_ERR_TIMEOUT = 6 when its consumers' bounded waits gave
        up); the solver stays usable."""
        return int(_lib.lib().pot3d_gpu_test_sweep_stall(self._h, spin_limit))

    def history(self, cap: int = 1 << 20) -> np.ndarray:
        """epsn after iterations 0..ncg of the last solve."""
        buf = np.zeros(cap)
        n = _lib.lib().pot3d_gpu_history(self._h, dptr(buf), cap)
        return buf[:n].copy()

    def finalize_phi(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        phi = np.zeros((self.mesh.nr, self.mesh.nt, self.mesh.np), order="F")
        check(_lib.lib().pot3d_gpu_finalize_phi(self._h, dptr(x), dptr(phi)))
        return phi

    def fields(self, x: np.ndarray, want=("phi", "br", "bt", "bp", "w")) -> dict:
        """phi, B and the magnetic energies from the interior solution x, one
        device call (potfld's finalisation, getb, magnetic_energy).  Returns
        the names in ``want``: phi (nr,nt,np), br (nrm1,nt,np),
        bt (nr,ntm1,np), bp (nr,nt,npm1), Fortran order; w = (W_r, W_t, W_p)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.size != self.N:
            raise ValueError(f"x has {x.size} values, the mesh has {self.N} unknowns")
        nr, nt, np_ = self.mesh.nr, self.mesh.nt, self.mesh.np
        shapes = {"phi": (nr, nt, np_), "br": (nr - 1, nt, np_), "bt": (nr, nt - 1, np_),
                  "bp": (nr, nt, np_ - 1), "w": (3,)}
        unknown = set(want) - set(shapes)
        if unknown:
            raise ValueError(f"unknown fields {sorted(unknown)}")
        out = {k: np.zeros(shapes[k], order="F") for k in want}
        ptr = [dptr(out[k]) if k in out else None for k in ("phi", "br", "bt", "bp", "w")]
        check(_lib.lib().pot3d_gpu_fields(self._h, dptr(x), *ptr))
        return out

    def energy(self, phi: np.ndarray) -> np.ndarray:
        phi = np.asfortranarray(phi, dtype=np.float64)
        w = np.zeros(3)
        check(_lib.lib().pot3d_gpu_energy(self._h, dptr(phi), dptr(w)))
        return w

    # ---- kernel-level entry points (device tensors) ---------------------
    def ax_dev(self, x, y):
        check(_lib.lib().pot3d_gpu_ax_dev(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())))

    def prec_dev(self, x):
        check(_lib.lib().pot3d_gpu_prec_dev(self._h, C.c_void_p(x.data_ptr())))

    def time_sweeps(self, reps: int = 10):
        """(forward ms, backward ms) of the ILU(0) wavefront sweeps (ifprec=2),
        in the form this solver iterates with (fused in the refined mode)."""
        ms = np.zeros(2)
        check(_lib.lib().pot3d_gpu_time_sweeps(self._h, reps, dptr(ms)))
        return float(ms[0]), float(ms[1])

    def time_kernels(self, reps: int = 20):
        """Average ms per launch of the stencil and update kernels, and their
        algorithmic DRAM bytes per launch."""
        ms = np.zeros(2)
        by = np.zeros(2)
        check(_lib.lib().pot3d_gpu_time_kernels(self._h, reps, dptr(ms), dptr(by)))
        return ms, by

    def precond_diag(self):
        d = np.zeros(self.N, np.float32)
        di = np.zeros(self.N, np.float32)
        check(_lib.lib().pot3d_gpu_precond_diag(self._h, fptr(d), fptr(di)))
        return d, di


def ernorm_lines(history, ncghist: int, epscg: float):
    """The convergence lines ernorm writes to pot3d.out
    (src/pot3d.F90:4435-4464): every ncghist iterations and the last one."""
    out = []
    n = len(history)
    for it in range(n):
        last = it == n - 1 and history[it] < epscg
        if (ncghist > 0 and it % ncghist == 0) or (last and ncghist > 0):
            out.append(f" Iteration: {it:8d}   Residual: {history[it]:23.15E}")
    return out


def potfld(mesh: Mesh, br0, option="ss", ifprec=1, precision="fp64", epscg=1e-9, ncgmax=10_000_000, x0=None):
    """The reference's potfld on the GPU: returns phi (with ghosts), the
    energies (W_r, W_t, W_p), iteration count, epsn and the history."""
    with Pot3dSolver(mesh, br0, option=option, ifprec=ifprec, precision=precision) as s:
        b = s.rhs()
        x = np.zeros(s.N) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        r = b.copy()
        ierr = s.cgsolve(x, r, ncgmax=ncgmax, epscg=epscg)
        info = s.last_info
        phi = s.finalize_phi(x)
        w = s.energy(phi)
        return dict(x=x, r=r, rhs=b, ierr=ierr, ncg=info.ncg, epsn=info.epsn, true_resid=info.true_resid,
                    seconds=info.seconds, n_refine=info.n_refine, launches=info.kernel_launches, phi=phi, energy=w,
                    history=s.history())


class BatchSolver:
    """Many independent PCG solves (own grid, Br map and outer radius each)
    advanced together by the batched kernels: every launch covers the tiles of
    all unfinished cases, each case stops at its own ernorm criterion.  FP64
    PCG with the diagonal preconditioner (ifprec=1) or ILU(0) (ifprec=2: both
    triangular sweeps of all cases run in one wavefront kernel per
    direction), FP64 or FP32-inner / FP64-refined (precision), from zero or
    from per-case guesses (set_guess).
    """

    def __init__(self, meshes, br0s, pm_r1s, tk: int = 0, ifprec: int = 1, precision: str = "fp64"):
        if not (len(meshes) == len(br0s) == len(pm_r1s)) or not meshes:
            raise ValueError("meshes, br0s and pm_r1s must be non-empty and of equal length")
        n = len(meshes)
        self.meshes = list(meshes)
        self._br = [np.asfortranarray(b, dtype=np.float64) for b in br0s]
        for m, b in zip(self.meshes, self._br):
            if b.shape != (m.nt, m.np):
                raise ValueError("br0 must have shape (nt, np) of its mesh")
        self._mcs = (_lib.MeshC * n)(*[m.cstruct() for m in self.meshes])
        self._keep = [m for m in self.meshes]  # keep mesh arrays alive
        self._brp = (C.POINTER(C.c_double) * n)(*[dptr(b) for b in self._br])
        self._r1 = np.ascontiguousarray(pm_r1s, dtype=np.float64)
        h = C.c_void_p()
        check(_lib.lib().pot3d_gpu_batch_create_mode(n, self._mcs, self._brp, dptr(self._r1), tk, ifprec,
                                                     PRECISION[precision], C.byref(h)))
        self._h = h
        self.n = n
        self.tk = tk
        self.ifprec = ifprec
        self.infos = None
        self.seconds = None

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().pot3d_gpu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def tune(self, candidates=(8, 16, 24, 32, 48, 64), iters: int = 6):
        """Pick the stencil's planes per block by timing; returns
        (best, {candidate: ms})."""
        c = (C.c_int * len(candidates))(*candidates)
        ms = (C.c_float * len(candidates))()
        best = C.c_int(0)
        check(_lib.lib().pot3d_gpu_batch_tune(self._h, c, len(candidates), iters, C.byref(best), ms))
        self.tk = best.value
        return best.value, {int(k): float(v) for k, v in zip(candidates, ms)}

    def tune2(self, candidates=(16, 32, 48, 64), update_candidates=(16, 32, 64, 128), iters: int = 6):
        """Pick the stencil's and the update kernels' planes per block
        together by timing every pair; returns ((best, best_update),
        {(candidate, update_candidate): ms})."""
        c = (C.c_int * len(candidates))(*candidates)
        d = (C.c_int * len(update_candidates))(*update_candidates)
        ms = (C.c_float * (len(candidates) * len(update_candidates)))()
        b, bu = C.c_int(0), C.c_int(0)
        check(_lib.lib().pot3d_gpu_batch_tune2(self._h, c, len(candidates), d, len(update_candidates), iters,
                                               C.byref(b), C.byref(bu), ms))
        self.tk = b.value
        times = {(int(x), int(y)): float(ms[i * len(update_candidates) + j])
                 for i, x in enumerate(candidates) for j, y in enumerate(update_candidates)}
        return (b.value, bu.value), times

    def solve(self, epscg: float = 1e-9, ncgmax: int = 10_000_000):
        """Solve every case; returns the list of ierr (0 = converged)."""
        ierr = (C.c_int * self.n)()
        infos = (SolveInfo * self.n)()
        sec = C.c_double(0.0)
        check(_lib.lib().pot3d_gpu_batch_solve(self._h, ncgmax, epscg, ierr, infos, C.byref(sec)))
        self.infos = list(infos)
        self.seconds = sec.value
        return list(ierr)

    def set_guess(self, i: int, x=None):
        """Initial guess of case i (packed layout, length N_i) for later
        solves; None returns to a zero guess."""
        if x is None:
            check(_lib.lib().pot3d_gpu_batch_set_guess(self._h, i, None))
            return
        m = self.meshes[i]
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.size != (m.nr - 2) * (m.nt - 2) * (m.np - 2):
            raise ValueError("guess has the wrong length for its case")
        check(_lib.lib().pot3d_gpu_batch_set_guess(self._h, i, dptr(x)))

    def solution(self, i: int) -> np.ndarray:
        """Interior solution of case i, packed layout (length N_i)."""
        m = self.meshes[i]
        x = np.zeros((m.nr - 2) * (m.nt - 2) * (m.np - 2))
        check(_lib.lib().pot3d_gpu_batch_solution(self._h, i, dptr(x)))
        return x
