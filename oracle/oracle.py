"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle (``pot3d_oracle.c``) restates POT3D's CPU PCG path from
src/pot3d.F90.  Only the test suite, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

OPTION_CODE = {"potential": 0, "open": 1, "ss": 2}
PM_R1 = {"potential": 1.0, "open": -1.0, "ss": -1.0}  # check_input, src/pot3d.F90:1250-1270


def build(force: bool = False) -> str:
    src = os.path.join(_HERE, "pot3d_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "CC=gcc"], check=True, capture_output=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        fp = C.POINTER(C.c_float)
        ip = C.POINTER(C.c_int)
        L.orc_genmesh.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, dp, dp, C.c_int, C.c_int, C.c_double, dp]
        L.orc_set_mesh.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, dp, dp, C.c_int, dp, dp, C.c_int,
                                   dp, dp, C.c_int, C.c_double]
        L.orc_readbr.argtypes = [C.c_void_p, C.c_int, C.c_int, dp, dp, dp, C.c_int, C.c_int, dp]
        L.orc_synthetic_br.argtypes = [C.c_ulonglong, C.c_int, C.c_int, C.c_int, C.c_int, dp, dp, dp]
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_void_p, dp, dp, C.c_double, C.c_int, ip]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_N.restype = C.c_long
        L.orc_N.argtypes = [C.c_void_p]
        L.orc_M.restype = C.c_long
        L.orc_M.argtypes = [C.c_void_p]
        L.orc_ilu_icode.argtypes = [C.c_void_p]
        L.orc_ax.argtypes = [C.c_void_p, dp, dp]
        L.orc_prec.argtypes = [C.c_void_p, dp]
        L.orc_lusol.argtypes = [C.c_void_p, fp]
        L.orc_rhs.argtypes = [C.c_void_p, dp]
        L.orc_cgsolve.argtypes = [C.c_void_p, dp, dp, C.c_int, C.c_double, C.c_int, ip, dp, ip, ip, dp, C.c_int]
        L.orc_finalize_phi.argtypes = [C.c_void_p, dp, dp]
        L.orc_energy.argtypes = [C.c_void_p, dp, dp]
        L.orc_getb.argtypes = [C.c_void_p, dp, dp, dp, dp]
        L.orc_get_ai.argtypes = [C.c_void_p, fp]
        L.orc_get_coef.argtypes = [C.c_void_p, dp]
        L.orc_get_ilu_diag.argtypes = [C.c_void_p, fp, fp]
        L.orc_build_csr.argtypes = [C.c_void_p, ip, ip, fp]
        L.orc_ilu0_csr.argtypes = [C.c_long, ip, ip, fp, ip]
        _lib = L
    return _lib


def _p(a, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct))


MESH_FIELDS = ("r", "dr", "rh", "drh", "t", "dt", "th", "dth", "st", "sth", "p", "dp", "ph", "dph")


class _MeshC(C.Structure):
    _fields_ = [("nr", C.c_int), ("nt", C.c_int), ("np", C.c_int)] + [(f, C.c_void_p) for f in MESH_FIELDS]


@dataclass
class Mesh:
    """1-D mesh arrays of one rank (Fortran element k is index k-1)."""

    nr: int
    nt: int
    np: int
    r: np.ndarray
    dr: np.ndarray
    rh: np.ndarray
    drh: np.ndarray
    t: np.ndarray
    dt: np.ndarray
    th: np.ndarray
    dth: np.ndarray
    st: np.ndarray
    sth: np.ndarray
    p: np.ndarray
    dp: np.ndarray
    ph: np.ndarray
    dph: np.ndarray

    def cstruct(self) -> _MeshC:
        s = _MeshC()
        s.nr, s.nt, s.np = self.nr, self.nt, self.np
        for f in MESH_FIELDS:
            setattr(s, f, getattr(self, f).ctypes.data)
        return s


def _seg(vals, nseg=30):
    a = np.zeros(nseg)
    v = np.atleast_1d(np.asarray(vals, dtype=np.float64))
    a[: v.size] = v
    return a


def genmesh(nc, c0, c1, frac, dratio, nfilt=0, periodic=False, c_shift=0.0):
    c = np.zeros(nc)
    f, d = _seg(frac), _seg(dratio)
    rc = lib().orc_genmesh(nc, c0, c1, 30, _p(f), _p(d), nfilt, int(periodic), c_shift, _p(c))
    if rc:
        raise ValueError(f"genmesh failed (code {rc})")
    return c


def make_mesh(nr, nt, np_, r0=1.0, r1=2.5, rfrac=(0.0, 1.0), drratio=(2.5,), nfrmesh=0, tfrac=(0.0,),
              dtratio=(1.0,), nftmesh=0, pfrac=(0.0,), dpratio=(1.0,), nfpmesh=0, phishift=0.0) -> Mesh:
    """set_global_mesh (src/pot3d.F90:2583-2708) at one rank."""
    m = Mesh(nr, nt, np_, np.zeros(nr - 1), np.zeros(nr - 1), np.zeros(nr), np.zeros(nr), np.zeros(nt - 1),
             np.zeros(nt - 1), np.zeros(nt), np.zeros(nt), np.zeros(nt - 1), np.zeros(nt), np.zeros(np_),
             np.zeros(np_), np.zeros(np_), np.zeros(np_))
    s = m.cstruct()
    args = [_seg(x) for x in (rfrac, drratio, tfrac, dtratio, pfrac, dpratio)]
    rc = lib().orc_set_mesh(C.byref(s), r0, r1, 30, _p(args[0]), _p(args[1]), nfrmesh, _p(args[2]),
                            _p(args[3]), nftmesh, _p(args[4]), _p(args[5]), nfpmesh, phishift)
    if rc:
        raise ValueError(f"set_global_mesh failed (code {rc})")
    return m


def readbr(mesh: Mesh, tn, pn, fi, option="ss", do_not_balance_flux=False) -> np.ndarray:
    """Interpolate a Br map fi[ntn, npn] (Fortran axis order) onto the mesh:
    readbr + set_flux (src/pot3d.F90:6672-6831, 3754-3864).  Returns br0 as
    a Fortran-ordered (nt, np) array."""
    fi = np.asfortranarray(np.asarray(fi, dtype=np.float64))
    tn = np.ascontiguousarray(tn, dtype=np.float64)
    pn = np.ascontiguousarray(pn, dtype=np.float64)
    br0 = np.zeros((mesh.nt, mesh.np), order="F")
    s = mesh.cstruct()
    rc = lib().orc_readbr(C.byref(s), fi.shape[0], fi.shape[1], _p(tn), _p(pn), _p(fi),
                          OPTION_CODE[option], int(do_not_balance_flux), _p(br0))
    if rc:
        raise ValueError(f"readbr failed (code {rc})")
    return br0


def synthetic_br(seed: int, lmax: int, nbip: int, ntn: int, npn: int):
    """Seeded synthetic Br map (tn, pn, fi[ntn, npn]); the product's
    generator restated, so a case can be built with the oracle alone."""
    tn, pn = np.zeros(ntn), np.zeros(npn)
    fi = np.zeros((ntn, npn), order="F")
    rc = lib().orc_synthetic_br(seed, lmax, nbip, ntn, npn, _p(tn), _p(pn), _p(fi))
    if rc:
        raise ValueError(f"synthetic_br failed (code {rc})")
    return tn, pn, fi


# Seeded workloads: grid and generator settings (the PFSS law r in [1, 2.5]).
WORKLOADS = {
    "pfss_63x91x181": dict(nr=63, nt=91, np=181, lmax=15, nbip=4, seed=1),
    "pfss_255x361x721": dict(nr=255, nt=361, np=721, lmax=40, nbip=20, seed=2),
    "pfss_127x181x361": dict(nr=127, nt=181, np=361, lmax=40, nbip=20, seed=1000),
}


def pfss_case(nr, nt, np_, lmax, nbip, seed, option="ss", do_not_balance_flux=False, r1=2.5):
    """(mesh, br0) of a seeded case built by the oracle alone."""
    mesh = make_mesh(nr, nt, np_, r1=r1)
    tn, pn, fi = synthetic_br(seed, lmax, nbip, nt, np_)
    return mesh, readbr(mesh, tn, pn, fi, option=option, do_not_balance_flux=do_not_balance_flux)


class Solver:
    """The solve context: coefficients + preconditioner (potfld set-up)."""

    def __init__(self, mesh: Mesh, br0, option="ss", ifprec=1, br1=None, pm_r1=None):
        self.mesh = mesh
        self._mesh_c = mesh.cstruct()
        self.br0 = np.asfortranarray(br0, dtype=np.float64)
        self.br1 = None if br1 is None else np.asfortranarray(br1, dtype=np.float64)
        pm = PM_R1[option] if pm_r1 is None else pm_r1
        st = C.c_int(0)
        self.h = lib().orc_create(C.byref(self._mesh_c), _p(self.br0),
                                  None if self.br1 is None else _p(self.br1), pm, ifprec, C.byref(st))
        self.status = st.value
        self.N = lib().orc_N(self.h)
        self.ifprec = ifprec

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def ax(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.N)
        lib().orc_ax(self.h, _p(x), _p(y))
        return y

    def prec(self, x):
        y = np.array(x, dtype=np.float64, copy=True)
        lib().orc_prec(self.h, _p(y))
        return y

    def lusol(self, x32):
        y = np.array(x32, dtype=np.float32, copy=True)
        lib().orc_lusol(self.h, _p(y, C.c_float))
        return y

    def rhs(self):
        b = np.zeros(self.N)
        lib().orc_rhs(self.h, _p(b))
        return b

    def a_i(self):
        a = np.zeros(self.N, np.float32)
        lib().orc_get_ai(self.h, _p(a, C.c_float))
        return a

    def coef(self):
        a = np.zeros(7 * self.N)
        lib().orc_get_coef(self.h, _p(a))
        return a.reshape(7, self.N)

    def ilu_diag(self):
        d = np.zeros(self.N, np.float32)
        di = np.zeros(self.N, np.float32)
        lib().orc_get_ilu_diag(self.h, _p(d, C.c_float), _p(di, C.c_float))
        return d, di

    def csr(self):
        """1-based CSR of A with boundary couplings dropped (getM + diacsr)."""
        N = self.N
        ia = np.zeros(N + 1, np.int32)
        # M from getM: IA(N+1) = nnz + 1
        tmp = Solver.__new__(Solver)
        nnz_bound = 7 * N
        ja = np.zeros(nnz_bound, np.int32)
        a = np.zeros(nnz_bound, np.float32)
        lib().orc_build_csr(self.h, _p(ia, C.c_int), _p(ja, C.c_int), _p(a, C.c_float))
        nnz = int(ia[-1]) - 1
        return ia, ja[:nnz].copy(), a[:nnz].copy()

    def cgsolve(self, x, r, ncgmax=10_000_000, epscg=1e-9, ncghist=0, hist_cap=100000):
        x = np.array(x, dtype=np.float64, copy=True)
        r = np.array(r, dtype=np.float64, copy=True)
        ncg = C.c_int(0)
        epsn = C.c_double(0)
        hn = C.c_int(0)
        hit = np.zeros(hist_cap, np.int32)
        heps = np.zeros(hist_cap)
        ierr = lib().orc_cgsolve(self.h, _p(x), _p(r), ncgmax, epscg, ncghist, C.byref(ncg), C.byref(epsn),
                                 C.byref(hn), _p(hit, C.c_int), _p(heps), hist_cap)
        hist = list(zip(hit[: hn.value].tolist(), heps[: hn.value].tolist()))
        return dict(x=x, r=r, ierr=ierr, ncg=ncg.value, epsn=epsn.value, history=hist)

    def finalize_phi(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        phi = np.zeros((self.mesh.nr, self.mesh.nt, self.mesh.np), order="F")
        lib().orc_finalize_phi(self.h, _p(x), _p(phi))
        return phi

    def energy(self, phi):
        phi = np.asfortranarray(phi, dtype=np.float64)
        w = np.zeros(3)
        lib().orc_energy(self.h, _p(phi), _p(w))
        return w

    def getb(self, phi):
        """(br, bt, bp) on the staggered meshes (src/pot3d.F90:6187-6233)."""
        phi = np.asfortranarray(phi, dtype=np.float64)
        nr, nt, np_ = self.mesh.nr, self.mesh.nt, self.mesh.np
        br = np.zeros((nr - 1, nt, np_), order="F")
        bt = np.zeros((nr, nt - 1, np_), order="F")
        bp = np.zeros((nr, nt, np_ - 1), order="F")
        lib().orc_getb(self.h, _p(phi), _p(br), _p(bt), _p(bp))
        return br, bt, bp


def ilu0_csr(ia, ja, a):
    """Reference ilu0 on a caller CSR (1-based), returns the factored values."""
    ia = np.ascontiguousarray(ia, np.int32)
    ja = np.ascontiguousarray(ja, np.int32)
    a = np.array(a, np.float32, copy=True)
    N = ia.size - 1
    dptr = np.zeros(N, np.int32)
    for i in range(N):
        cols = ja[ia[i] - 1: ia[i + 1] - 1]
        dptr[i] = ia[i] + int(np.nonzero(cols == i + 1)[0][0])
    icode = lib().orc_ilu0_csr(N, _p(ia, C.c_int), _p(ja, C.c_int), _p(a, C.c_float), _p(dptr, C.c_int))
    return a, icode


def potfld(mesh: Mesh, br0, option="ss", ifprec=1, epscg=1e-9, ncgmax=10_000_000, ncghist=0, x0=None):
    """Full reference-path solve: RHS, PCG, phi with ghosts and energies."""
    s = Solver(mesh, br0, option=option, ifprec=ifprec)
    if s.status:
        raise RuntimeError(f"preconditioner set-up failed (code {s.status})")
    b = s.rhs()
    x = np.zeros(s.N) if x0 is None else x0
    out = s.cgsolve(x, b, ncgmax=ncgmax, epscg=epscg, ncghist=ncghist)
    phi = s.finalize_phi(out["x"])
    out["phi"] = phi
    out["energy"] = s.energy(phi)
    out["rhs"] = b
    return out


def threads() -> int:
    return lib().orc_threads()
