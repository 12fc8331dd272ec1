"""GPU parity of the ILU(0) preconditioner (ifprec=2) against the oracle.

The factor (U diagonal and its FP32 inverse) and one application of the
preconditioner are compared bit for bit: both follow ilu0/lusol operation
for operation in FP32 without fused multiply-adds.  Solves are compared at
epscg 1e-11 (phi relative L2 <= 1e-8, energies <= 1e-9 relative).  The
legacy external-LU symbols are driven through ctypes with device pointers,
as the Fortran host calls them.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from pot3d_b200 import _lib, host
from pot3d_b200.solver import Pot3dSolver, potfld

pytestmark = pytest.mark.gpu

GRIDS = [(12, 11, 14), (37, 30, 26), (20, 13, 11), (9, 7, 8), (70, 45, 90)]


def _case(nr, nt, np_, seed=3, option="ss"):
    mesh = host.make_mesh(nr, nt, np_)
    tn, pn, fi = host.synthetic_br(seed, 15, 4, nt, np_)
    return mesh, host.br0_from_map(mesh, tn, pn, fi, option=option)


def _oracle(mesh, br0, option="ss", ifprec=2):
    mo = O.Mesh(mesh.nr, mesh.nt, mesh.np, *[getattr(mesh, f) for f in O.MESH_FIELDS])
    return O.Solver(mo, br0, option, ifprec)


@pytest.mark.parametrize("dims", GRIDS)
def test_dilu_factor_and_apply_bitwise(cuda, dims):
    import torch
    mesh, br0 = _case(*dims)
    o = _oracle(mesh, br0)
    with Pot3dSolver(mesh, br0, ifprec=2) as s:
        d, dinv = s.precond_diag()
        d_ref, dinv_ref = o.ilu_diag()
        assert np.array_equal(d, d_ref)
        assert np.array_equal(dinv, dinv_ref)
        x = np.random.default_rng(7).standard_normal(s.N)
        xt = torch.tensor(x, device=cuda)
        s.prec_dev(xt)
        z = xt.cpu().numpy()
        assert np.array_equal(z, o.prec(x))
        # the sweeps' tile counters and tags carry over between applications
        for _ in range(3):
            xt = torch.tensor(x, device=cuda)
            s.prec_dev(xt)
            assert np.array_equal(xt.cpu().numpy(), z)


@pytest.mark.parametrize("dims,option", [((37, 30, 26), "ss"), ((20, 13, 11), "open")])
def test_ilu_solve_parity_at_1e11(cuda, dims, option):
    mesh, br0 = _case(*dims, option=option)
    o = _oracle(mesh, br0, option=option)
    ref = o.cgsolve(np.zeros(o.N), o.rhs(), epscg=1e-11)
    phi_ref = o.finalize_phi(ref["x"])
    w_ref = o.energy(phi_ref)
    out = potfld(mesh, br0, option=option, ifprec=2, epscg=1e-11)
    assert out["ierr"] == 0
    rel = np.linalg.norm(out["phi"] - phi_ref) / np.linalg.norm(phi_ref)
    assert rel <= 1e-8, rel
    assert np.all(np.abs(out["energy"] - w_ref) <= 1e-9 * np.abs(w_ref))
    assert abs(out["ncg"] - ref["ncg"]) <= max(2, ref["ncg"] // 50)
    # ILU(0) needs fewer iterations than the diagonal preconditioner
    diag = potfld(mesh, br0, option=option, ifprec=1, epscg=1e-11)
    assert out["ncg"] < diag["ncg"]


def _legacy():
    L = _lib.lib()
    return L.load_external_lu_solver, L.external_lu_solver, L.unload_external_lu_solver


@pytest.mark.parametrize("dims", [(12, 11, 14), (30, 21, 17), (63, 91, 181)])
def test_legacy_external_lu_solver(cuda, dims):
    """load/external/unload_external_lu_solver on device CSR arrays built by
    the oracle's getM/diacsr, as the -DCUSPARSE Fortran host passes them."""
    import torch
    mesh, br0 = _case(*dims)
    o = _oracle(mesh, br0)
    ia, ja, a = o.csr()
    f_ref, icode = O.ilu0_csr(ia, ja, a)
    assert icode == 0
    load, apply_, unload = _legacy()
    for _round in range(2):  # load / use / unload twice
        ia_d = torch.tensor(ia, dtype=torch.int32, device=cuda)
        ja_d = torch.tensor(ja, dtype=torch.int32, device=cuda)
        a_d = torch.tensor(a, dtype=torch.float32, device=cuda)
        torch.cuda.synchronize()
        load(C.c_void_p(a_d.data_ptr()), C.c_void_p(ia_d.data_ptr()), C.c_void_p(ja_d.data_ptr()), o.N,
             int(ia[-1]))
        assert np.array_equal(a_d.cpu().numpy(), f_ref)  # factorised in place, bit for bit
        rng = np.random.default_rng(_round)
        for _ in range(2):
            x = rng.standard_normal(o.N)
            xt = torch.tensor(x, device=cuda)
            apply_(C.c_void_p(xt.data_ptr()))
            assert np.array_equal(xt.cpu().numpy(), o.prec(x))
        unload()


def _apply(load, apply_, unload, ia, ja, a, N, rhs, cuda):
    import torch
    ia_d = torch.tensor(ia, dtype=torch.int32, device=cuda)
    ja_d = torch.tensor(ja, dtype=torch.int32, device=cuda)
    a_d = torch.tensor(a, dtype=torch.float32, device=cuda)
    torch.cuda.synchronize()
    load(C.c_void_p(a_d.data_ptr()), C.c_void_p(ia_d.data_ptr()), C.c_void_p(ja_d.data_ptr()), N, int(ia[-1]))
    xt = torch.tensor(rhs, device=cuda)
    apply_(C.c_void_p(xt.data_ptr()))
    z = xt.cpu().numpy()
    unload()
    return z


def _lusol_np(ia, ja, lu, x):
    """lusol (src/pot3d.F90:5227-5302) on a general factored 1-based CSR in
    FP32, one rounding per operation; dinv = real(1/d in FP64, REAL32)."""
    N = ia.size - 1
    y = x.astype(np.float32)
    f = np.float32
    diag = [int(np.nonzero(ja[ia[i] - 1:ia[i + 1] - 1] == i + 1)[0][0]) + ia[i] - 1 for i in range(N)]
    for i in range(N):
        v = y[i]
        for k in range(ia[i] - 1, diag[i]):
            v = f(v - f(lu[k] * y[ja[k] - 1]))
        y[i] = v
    for i in range(N - 1, -1, -1):
        v = y[i]
        for k in range(diag[i] + 1, ia[i + 1] - 1):
            v = f(v - f(lu[k] * y[ja[k] - 1]))
        y[i] = f(v * np.float32(1.0 / np.float64(lu[diag[i]])))
    return y.astype(np.float64)


def test_legacy_general_pattern_uses_the_level_route(cuda):
    """A CSR without the 7-point pattern (random structurally symmetric,
    diagonally dominant) goes through the level-scheduled sweeps; the
    factor is ilu0's and the solve lusol's, bit for bit."""
    rng = np.random.default_rng(9)
    N = 300
    rows = [set([i]) for i in range(N)]
    for _ in range(4 * N):
        i, j = rng.integers(N, size=2)
        rows[i].add(int(j))
        rows[j].add(int(i))
    ia, ja, a = [1], [], []
    for i in range(N):
        cols = sorted(rows[i])
        for j in cols:
            ja.append(j + 1)
            a.append(float(len(cols) + 1) if j == i else float(rng.uniform(-1, 0)))
        ia.append(len(ja) + 1)
    ia = np.array(ia, np.int32)
    ja = np.array(ja, np.int32)
    a = np.array(a, np.float32)
    f_ref, icode = O.ilu0_csr(ia, ja, a)
    assert icode == 0
    rhs = rng.standard_normal(N)
    z = _apply(*_legacy(), ia, ja, a, N, rhs, cuda)
    assert np.array_equal(z, _lusol_np(ia, ja, f_ref, rhs))
