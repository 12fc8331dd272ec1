"""readbr on the device (pot3d_gpu_br0_from_map) against the host readbr
(itself bit for bit the oracle's restatement of src/pot3d.F90:6672-6831):
the reference test suite's Br maps on their meshes and seeded synthetic
maps, every option, with and without flux balance -- bit for bit -- and the
solve that follows it equals the one set up from the host's br0."""
import numpy as np
import pytest

from conftest import CASES, load_case
from pot3d_b200 import host
from pot3d_b200._lib import Pot3dError
from pot3d_b200.solver import Pot3dSolver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", CASES)
def test_testsuite_maps_bitwise(cuda, case):
    meta, z = load_case(case)
    nml = meta["namelist"]
    m = host.make_mesh(nml["nr"], nml["nt"], nml["np"], r0=nml["r0"], r1=nml["r1"], rfrac=nml["rfrac"],
                       drratio=nml["drratio"], nfrmesh=nml["nfrmesh"], tfrac=nml["tfrac"], dtratio=nml["dtratio"],
                       nftmesh=nml["nftmesh"], pfrac=nml["pfrac"], dpratio=nml["dpratio"], nfpmesh=nml["nfpmesh"],
                       phishift=nml["phishift"])
    fi = np.asarray(z["data"], np.float64)
    ref = host.br0_from_map(m, z["tn"], z["pn"], fi, nml["option"], nml["do_not_balance_flux"])
    with Pot3dSolver(m, np.zeros((m.nt, m.np), order="F"), option=nml["option"]) as s:
        got = s.br0_from_map(z["tn"], z["pn"], fi, nml["option"], nml["do_not_balance_flux"])
        assert np.array_equal(got, ref)
        b_dev = s.rhs()
    with Pot3dSolver(m, ref, option=nml["option"]) as s2:
        assert np.array_equal(b_dev, s2.rhs())


@pytest.mark.parametrize("option,dnb", [("ss", False), ("open", True), ("open", False), ("potential", False)])
def test_synthetic_maps_bitwise_and_solve(cuda, option, dnb):
    mesh = host.make_mesh(37, 30, 26)
    tn, pn, fi = host.synthetic_br(21, 15, 4, 45, 61)  # a map on its own (finer) grid
    ref = host.br0_from_map(mesh, tn, pn, fi, option, dnb)
    with Pot3dSolver(mesh, np.zeros((mesh.nt, mesh.np), order="F"), option=option) as s:
        got = s.br0_from_map(tn, pn, fi, option, dnb)
        assert np.array_equal(got, ref)
        x = np.zeros(s.N)
        r = s.rhs()
        assert s.cgsolve(x, r, epscg=1e-10) == 0
    with Pot3dSolver(mesh, ref, option=option) as s2:
        x2 = np.zeros(s2.N)
        r2 = s2.rhs()
        assert s2.cgsolve(x2, r2, epscg=1e-10) == 0
    assert np.array_equal(x, x2)


def test_bad_scales_are_rejected(cuda):
    mesh = host.make_mesh(20, 13, 11)
    tn, pn, fi = host.synthetic_br(2, 5, 0, 13, 11)
    with Pot3dSolver(mesh, np.zeros((mesh.nt, mesh.np), order="F")) as s:
        with pytest.raises(Pot3dError):
            s.br0_from_map(tn[::-1].copy(), pn, fi)
        with pytest.raises(Pot3dError):  # a map that does not reach the poles
            s.br0_from_map(tn[1:-1].copy(), pn, fi[1:-1])
