"""Failure detection on the GPU without a fault: every device wait of the
library is bounded and ends in a status code the host reads.

* A wavefront sweep with one tile left undone: the tiles that consume its
  faces wait for words nobody publishes; with a short poll limit the waits
  give up, the call returns POT3D_ERR_TIMEOUT within a second, and the next
  solve on the same handle is correct (the context stays usable).
* A boundary map with a NaN: the PCG state reports a breakdown
  (POT3D_ERR_BREAKDOWN) in both arithmetic modes instead of iterating to
  ncgmax, and the handle solves again once a finite map is set.
"""
import time

import numpy as np
import pytest

import oracle as O
from pot3d_b200 import host
from pot3d_b200._lib import Pot3dError
from pot3d_b200.solver import Pot3dSolver

pytestmark = pytest.mark.gpu

POT3D_ERR_TIMEOUT = 6
POT3D_ERR_BREAKDOWN = 7


def _case(nr, nt, np_, seed=3):
    mesh = host.make_mesh(nr, nt, np_)
    tn, pn, fi = host.synthetic_br(seed, 15, 4, nt, np_)
    return mesh, host.br0_from_map(mesh, tn, pn, fi)


def _oracle_x(mesh, br0, ifprec):
    mo = O.Mesh(mesh.nr, mesh.nt, mesh.np, *[getattr(mesh, f) for f in O.MESH_FIELDS])
    o = O.Solver(mo, br0, "ss", ifprec)
    return o.cgsolve(np.zeros(o.N), o.rhs(), epscg=1e-11)["x"]


@pytest.mark.parametrize("dims", [(37, 30, 26), (63, 91, 181)])
def test_sweep_wait_runs_out_and_the_solver_recovers(dims):
    mesh, br0 = _case(*dims)
    with Pot3dSolver(mesh, br0, ifprec=2) as s:
        t0 = time.perf_counter()
        rc = s.test_sweep_stall(1 << 12)
        assert rc == POT3D_ERR_TIMEOUT
        assert time.perf_counter() - t0 < 2.0
        # same handle, next solve: converges to the oracle's solution
        b = s.rhs()
        x = np.zeros(s.N)
        r = b.copy()
        assert s.cgsolve(x, r, epscg=1e-11, ncgmax=20000) == 0
    ref = _oracle_x(mesh, br0, 2)
    assert np.linalg.norm(x - ref) <= 1e-8 * np.linalg.norm(ref)


@pytest.mark.parametrize("ifprec,precision", [(1, "fp64"), (2, "fp64"), (2, "fp32_refined"), (1, "fp32_refined")])
def test_nan_boundary_map_reports_breakdown(ifprec, precision):
    mesh, br0 = _case(20, 13, 11)
    bad = br0.copy()
    bad[5, 4] = np.nan
    with Pot3dSolver(mesh, bad, ifprec=ifprec, precision=precision) as s:
        b = s.rhs()
        assert np.isnan(b).any()
        x = np.zeros(s.N)
        r = b.copy()
        with pytest.raises(Pot3dError) as ei:
            s.cgsolve(x, r, epscg=1e-11, ncgmax=20000)
        assert ei.value.code == POT3D_ERR_BREAKDOWN
        # a finite map on the same handle solves again
        s.set_br0(br0)
        b = s.rhs()
        x = np.zeros(s.N)
        r = b.copy()
        assert s.cgsolve(x, r, epscg=1e-11, ncgmax=20000) == 0
    ref = _oracle_x(mesh, br0, ifprec)
    assert np.linalg.norm(x - ref) <= 1e-8 * np.linalg.norm(ref)


def test_stall_hook_rejects_bad_arguments():
    mesh, br0 = _case(20, 13, 11)
    with Pot3dSolver(mesh, br0, ifprec=1) as s:
        assert s.test_sweep_stall(1 << 12) == 1  # POT3D_ERR_ARG: no sweeps with the diagonal preconditioner
