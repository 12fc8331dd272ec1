"""Host-side inputs of the solve: meshes, boundary maps, synthetic Br.

Thin Python front end of include/pot3d_host.h.  The mesh is the set of 1-D
arrays POT3D's set_global_mesh (src/pot3d.F90:2583-2708) produces at one
rank; br0 is what readbr/set_flux (src/pot3d.F90:6672-6831, 3754-3864)
leave in the module array br0(nt,np).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import MESH_FIELDS, dptr

NSEG = 30
OPTION_CODE = {"potential": 0, "open": 1, "ss": 2}
PM_R1 = {"potential": 1.0, "open": -1.0, "ss": -1.0}


@dataclass
class Mesh:
    nr: int
    nt: int
    np: int
    r: np.ndarray
    dr: np.ndarray
    rh: np.ndarray
    drh: np.ndarray
    t: np.ndarray
    dt: np.ndarray
    st: np.ndarray
    th: np.ndarray
    dth: np.ndarray
    sth: np.ndarray
    p: np.ndarray
    dp: np.ndarray
    ph: np.ndarray
    dph: np.ndarray

    def cstruct(self) -> _lib.MeshC:
        s = _lib.MeshC()
        s.nr, s.nt, s.np = self.nr, self.nt, self.np
        for f in MESH_FIELDS:
            a = getattr(self, f)
            assert a.dtype == np.float64 and a.flags.c_contiguous
            setattr(s, f, a.ctypes.data)
        return s

    @classmethod
    def empty(cls, nr, nt, np_):
        z = np.zeros
        return cls(nr, nt, np_, z(nr - 1), z(nr - 1), z(nr), z(nr), z(nt - 1), z(nt - 1), z(nt - 1), z(nt), z(nt),
                   z(nt), z(np_), z(np_), z(np_), z(np_))

    @property
    def N(self) -> int:
        return (self.nr - 2) * (self.nt - 2) * (self.np - 2)


def _seg(vals):
    a = np.zeros(NSEG)
    v = np.atleast_1d(np.asarray(vals, dtype=np.float64))
    a[: v.size] = v
    return a


def genmesh(nc, c0, c1, frac, dratio, nfilt=0, periodic=False, c_shift=0.0) -> np.ndarray:
    c = np.zeros(nc)
    f, d = _seg(frac), _seg(dratio)
    rc = _lib.lib().pot3d_host_genmesh(nc, c0, c1, NSEG, dptr(f), dptr(d), nfilt, int(periodic), c_shift, dptr(c))
    if rc:
        raise ValueError(f"genmesh failed (code {rc})")
    return c


def make_mesh(nr, nt, np_, r0=1.0, r1=2.5, rfrac=(0.0, 1.0), drratio=(2.5,), nfrmesh=0, tfrac=(0.0,),
              dtratio=(1.0,), nftmesh=0, pfrac=(0.0,), dpratio=(1.0,), nfpmesh=0, phishift=0.0) -> Mesh:
    """Mesh of set_global_mesh; defaults are the PFSS law r in [1,2.5],
    drratio 2.5, uniform theta and phi."""
    m = Mesh.empty(nr, nt, np_)
    s = m.cstruct()
    a = [_seg(x) for x in (rfrac, drratio, tfrac, dtratio, pfrac, dpratio)]
    rc = _lib.lib().pot3d_host_mesh(s, r0, r1, NSEG, dptr(a[0]), dptr(a[1]), nfrmesh, dptr(a[2]), dptr(a[3]),
                                    nftmesh, dptr(a[4]), dptr(a[5]), nfpmesh, phishift)
    if rc:
        raise ValueError(f"set_global_mesh failed (code {rc})")
    return m


def mesh_from_namelist(nml) -> Mesh:
    v = nml if isinstance(nml, dict) else nml.values
    return make_mesh(v["nr"], v["nt"], v["np"], r0=v["r0"], r1=v["r1"], rfrac=v["rfrac"], drratio=v["drratio"],
                     nfrmesh=v["nfrmesh"], tfrac=v["tfrac"], dtratio=v["dtratio"], nftmesh=v["nftmesh"],
                     pfrac=v["pfrac"], dpratio=v["dpratio"], nfpmesh=v["nfpmesh"], phishift=v["phishift"])


def br0_from_map(mesh: Mesh, tn, pn, fi, option="ss", do_not_balance_flux=False) -> np.ndarray:
    """readbr + set_flux: interpolate fi[ntn,npn] (Fortran axis order) to
    the mesh.  Returns br0 as a Fortran-ordered (nt, np) array."""
    fi = np.asfortranarray(np.asarray(fi, dtype=np.float64))
    tn = np.ascontiguousarray(tn, dtype=np.float64)
    pn = np.ascontiguousarray(pn, dtype=np.float64)
    br0 = np.zeros((mesh.nt, mesh.np), order="F")
    rc = _lib.lib().pot3d_host_br0(mesh.cstruct(), fi.shape[0], fi.shape[1], dptr(tn), dptr(pn), dptr(fi),
                                   OPTION_CODE[option], int(do_not_balance_flux), dptr(br0))
    if rc:
        raise ValueError(f"readbr failed (code {rc})")
    return br0


def synthetic_br(seed: int, lmax: int, nbip: int, ntn: int, npn: int):
    """Seeded synthetic Br map; returns (tn, pn, fi[ntn, npn])."""
    tn, pn = np.zeros(ntn), np.zeros(npn)
    fi = np.zeros((ntn, npn), order="F")
    rc = _lib.lib().pot3d_host_synthetic_br(seed, lmax, nbip, ntn, npn, dptr(tn), dptr(pn), dptr(fi))
    if rc:
        raise ValueError(f"synthetic_br failed (code {rc})")
    return tn, pn, fi


# Workloads named by grid size and generator settings.
WORKLOADS = {
    "pfss_63x91x181": dict(nr=63, nt=91, np=181, lmax=15, nbip=4, seed=1),
    "pfss_255x361x721": dict(nr=255, nt=361, np=721, lmax=40, nbip=20, seed=2),
    "pfss_255x361x181": dict(nr=255, nt=361, np=181, lmax=40, nbip=20, seed=2),
    "pfss_127x181x361": dict(nr=127, nt=181, np=361, lmax=40, nbip=20, seed=1000),
    "open_511x721x1441": dict(nr=511, nt=721, np=1441, lmax=80, nbip=60, seed=7, option="open",
                              do_not_balance_flux=True),
}


def pfss_case(nr, nt, np_, lmax, nbip, seed, option="ss", do_not_balance_flux=False, r1=2.5):
    """Mesh and br0 of a seeded PFSS (or open) case on the PFSS grid law."""
    mesh = make_mesh(nr, nt, np_, r1=r1)
    tn, pn, fi = synthetic_br(seed, lmax, nbip, nt, np_)
    br0 = br0_from_map(mesh, tn, pn, fi, option=option, do_not_balance_flux=do_not_balance_flux)
    return mesh, br0


def _seq_sum(a) -> float:
    """Left-to-right sum (the order of a serial Fortran SUM)."""
    s = 0.0
    for v in np.asarray(a, dtype=np.float64).ravel():
        s += float(v)
    return s


def validation_br(mesh: Mesh, dipole_angle: float, r0: float, r1: float):
    """set_validation_flux (src/pot3d.F90:3978-4066): the tilted-dipole Br at
    r0 and r1 on the (nt, np) half mesh, periodic in phi, with the pole ghost
    rows set from the m=0 average.  Returns (br0, br1), Fortran order."""
    cth, sth, cph = np.cos(mesh.th), np.sin(mesh.th), np.cos(mesh.ph)
    ca, sa = np.cos(dipole_angle), np.sin(dipole_angle)
    pl_i = 1.0 / (2.0 * 3.1415926535897932 - 0.0)
    nt, np_ = mesh.nt, mesh.np
    out = []
    for rr in (r0, r1):
        b = np.asfortranarray((2.0 / (rr * rr * rr)) * (cth[:, None] * ca + (sth[:, None] * cph[None, :]) * sa))
        b[:, 0] = b[:, np_ - 2]
        b[:, np_ - 1] = b[:, 1]
        s00 = _seq_sum(b[1, 1:np_ - 1] * mesh.dph[1:np_ - 1]) * pl_i
        s11 = _seq_sum(b[nt - 2, 1:np_ - 1] * mesh.dph[1:np_ - 1]) * pl_i
        b[0, :] = 2.0 * s00 - b[1, :]
        b[nt - 1, :] = 2.0 * s11 - b[nt - 2, :]
        out.append(b)
    return out[0], out[1]


def _seam_phi(a):
    """seam_gen in the periodic dimension at one rank (src/pot3d.F90:5846-6013)."""
    n3 = a.shape[2]
    a[:, :, 0] = a[:, :, n3 - 2]
    a[:, :, n3 - 1] = a[:, :, 1]
    return a


def validation_exact(mesh: Mesh, dipole_angle: float):
    """The analytic tilted-dipole solution of write_validation_solution
    (src/pot3d.F90:4068-4131): phi's interior values (packed, length N; the
    ghosts follow from the boundary conditions as in the reference) and
    br (nrm1,nt,np), bt (nr,ntm1,np), bp (nr,nt,npm1) on the staggered
    meshes, seamed in phi."""
    ca, sa = np.cos(dipole_angle), np.sin(dipole_angle)
    nr, nt, np_ = mesh.nr, mesh.nt, mesh.np
    cth, sth = np.cos(mesh.th), np.sin(mesh.th)
    ct, st = np.cos(mesh.t), np.sin(mesh.t)
    cph, sph = np.cos(mesh.ph), np.sin(mesh.ph)
    ang_h = cth[:, None] * ca + (sth[:, None] * cph[None, :]) * sa          # (nt, np)
    phi = (-1.0 / (mesh.rh * mesh.rh))[:, None, None] * ang_h[None]
    x = np.ascontiguousarray(phi[1:-1, 1:-1, 1:-1].transpose(2, 1, 0)).ravel()
    br = (2.0 / (mesh.r * mesh.r * mesh.r))[:, None, None] * ang_h[None]
    bt = (1.0 / (mesh.rh * mesh.rh * mesh.rh))[:, None, None] * (st[:, None] * ca - (ct[:, None] * cph[None, :]) * sa)[None]
    # the reference evaluates bp with the half-mesh sin(ph(k))
    bp = (1.0 / (mesh.rh * mesh.rh * mesh.rh))[:, None, None] * np.broadcast_to(sph[None, None, :np_ - 1] * sa, (1, nt, np_ - 1))
    return (x, _seam_phi(np.asfortranarray(br)), _seam_phi(np.asfortranarray(bt)),
            _seam_phi(np.asfortranarray(bp)))
