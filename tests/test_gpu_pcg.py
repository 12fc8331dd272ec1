"""GPU parity of the FP64 PCG path against the oracle, through the C-ABI.

Tolerances: coefficient-identical kernels (RHS, the FP32 diagonal
preconditioner, phi finalisation) are compared bit for bit; the stencil is
compared to 1e-13 of the largest term (its seven products are summed with
FMAs on the GPU, separately rounded in the oracle); solves are compared at
epscg 1e-11 with phi to relative L2 <= 1e-8 and energies to <= 1e-9
relative, and on the reference test-suite cases the energies must round to
the reference's values at 7 decimals (bin/pot3d_validation.sh).
"""
import numpy as np
import pytest

import oracle as O
from conftest import CASES, load_case
from pot3d_b200 import host
from pot3d_b200.solver import Pot3dSolver, potfld

pytestmark = pytest.mark.gpu

GRIDS = [(63, 91, 181), (20, 13, 11), (37, 30, 26), (70, 23, 19)]


def _case(nr, nt, np_, seed=1, option="ss"):
    mesh = host.make_mesh(nr, nt, np_)
    tn, pn, fi = host.synthetic_br(seed, 15, 4, nt, np_)
    br0 = host.br0_from_map(mesh, tn, pn, fi, option=option)
    return mesh, br0


def _oracle(mesh, br0, option="ss", ifprec=1):
    mo = O.Mesh(mesh.nr, mesh.nt, mesh.np, *[getattr(mesh, f) for f in O.MESH_FIELDS])
    return O.Solver(mo, br0, option, ifprec)


@pytest.mark.parametrize("dims", GRIDS)
def test_stencil_matches_oracle(cuda, dims):
    import torch
    mesh, br0 = _case(*dims)
    s = Pot3dSolver(mesh, br0)
    o = _oracle(mesh, br0)
    rng = np.random.default_rng(5)
    for _ in range(2):
        x = rng.standard_normal(s.N)
        y_ref = o.ax(x)
        xt = torch.tensor(x, device=cuda)
        yt = torch.empty_like(xt)
        s.ax_dev(xt, yt)
        y = yt.cpu().numpy()
        coef = np.abs(o.coef())
        scale = np.max(coef.sum(axis=0)) * np.max(np.abs(x))
        assert np.max(np.abs(y - y_ref)) <= 1e-13 * scale


@pytest.mark.parametrize("dims", GRIDS[:2])
def test_rhs_and_diag_preconditioner_bitwise(cuda, dims):
    mesh, br0 = _case(*dims)
    s = Pot3dSolver(mesh, br0)
    o = _oracle(mesh, br0)
    assert np.array_equal(s.rhs(), o.rhs())
    d, _ = s.precond_diag()
    assert np.array_equal(d, o.a_i())


def test_prec_apply_matches_oracle(cuda):
    import torch
    mesh, br0 = _case(37, 30, 26)
    s = Pot3dSolver(mesh, br0)
    o = _oracle(mesh, br0)
    x = np.random.default_rng(3).standard_normal(s.N)
    xt = torch.tensor(x, device=cuda)
    s.prec_dev(xt)
    assert np.array_equal(xt.cpu().numpy(), o.prec(x))


@pytest.mark.parametrize("dims,option", [((63, 91, 181), "ss"), ((37, 30, 26), "open"), ((20, 13, 11), "potential")])
def test_solve_parity_at_1e11(cuda, dims, option):
    mesh, br0 = _case(*dims, option=option)
    o = _oracle(mesh, br0, option=option)
    ref = o.cgsolve(np.zeros(o.N), o.rhs(), epscg=1e-11)
    phi_ref = o.finalize_phi(ref["x"])
    w_ref = o.energy(phi_ref)
    out = potfld(mesh, br0, option=option, epscg=1e-11)
    assert out["ierr"] == 0
    rel = np.linalg.norm(out["phi"] - phi_ref) / np.linalg.norm(phi_ref)
    assert rel <= 1e-8, rel
    assert np.all(np.abs(out["energy"] - w_ref) <= 1e-9 * np.abs(w_ref))
    assert abs(out["ncg"] - ref["ncg"]) <= max(3, ref["ncg"] // 100)
    assert out["true_resid"] < 1e-8


def test_finalize_and_energy_match_oracle(cuda):
    mesh, br0 = _case(37, 30, 26)
    s = Pot3dSolver(mesh, br0)
    o = _oracle(mesh, br0)
    x = np.random.default_rng(9).standard_normal(s.N)
    phi = s.finalize_phi(x)
    phi_ref = o.finalize_phi(x)
    assert np.array_equal(phi, phi_ref)
    w, w_ref = s.energy(phi), o.energy(phi_ref)
    assert np.all(np.abs(w - w_ref) <= 1e-12 * np.abs(w_ref))


@pytest.mark.parametrize("dims", [(37, 30, 26), (20, 13, 11), (9, 7, 8)])
def test_fields_getb_bitwise(cuda, dims):
    """phi, br, bt, bp of the one-call post-solve path equal the oracle's
    getb bit for bit; the energies agree to 1e-12 (summation order)."""
    mesh, br0 = _case(*dims)
    s = Pot3dSolver(mesh, br0)
    o = _oracle(mesh, br0)
    x = np.random.default_rng(11).standard_normal(s.N)
    out = s.fields(x)
    phi_ref = o.finalize_phi(x)
    assert np.array_equal(out["phi"], phi_ref)
    for got, ref in zip((out["br"], out["bt"], out["bp"]), o.getb(phi_ref)):
        assert got.shape == ref.shape
        assert np.array_equal(got, ref)
    w_ref = o.energy(phi_ref)
    assert np.all(np.abs(out["w"] - w_ref) <= 1e-12 * np.abs(w_ref))
    # subsets: only what is asked for is returned, and it is the same
    part = s.fields(x, want=("bt", "w"))
    assert set(part) == {"bt", "w"}
    assert np.array_equal(part["bt"], out["bt"])
    assert np.array_equal(part["w"], out["w"])
    with pytest.raises(ValueError):
        s.fields(x[:-1])


@pytest.mark.parametrize("case", CASES)
def test_reference_testsuite_energies(cuda, case):
    """The three cases of POT3D's test suite, solved on the GPU: energies
    match the reference's pot3d.out at 7 decimals (the suite's criterion),
    and the iteration count and the logged residual history agree."""
    meta, z = load_case(case)
    nml = meta["namelist"]
    ref = meta["reference"]
    mesh = host.mesh_from_namelist(nml)
    br0 = host.br0_from_map(mesh, z["tn"], z["pn"], np.asarray(z["data"], np.float64), nml["option"],
                            nml["do_not_balance_flux"])
    out = potfld(mesh, br0, option=nml["option"], ifprec=nml["ifprec"], epscg=nml["epscg"])
    assert out["ierr"] == 0
    for val, key in zip(out["energy"], ("wr", "wt", "wp")):
        assert round(val, 7) == round(ref["energy"][key], 7), key
        assert abs(val - ref["energy"][key]) <= 1e-9 * abs(ref["energy"][key])
    assert abs(out["ncg"] - ref["iterations"]) <= 2
    h = out["history"]
    for it, e in ref["history"]:
        if it < len(h):
            assert abs(h[it] - e) <= 1e-6 * e, (it, h[it], e)


def test_zero_rhs_and_ncgmax(cuda):
    mesh, br0 = _case(20, 13, 11)
    with Pot3dSolver(mesh, np.zeros_like(br0)) as s:
        x = np.ones(s.N)
        r = np.zeros(s.N)
        assert s.cgsolve(x, r) == 0
        assert not x.any() and s.last_info.ncg == 0
    with Pot3dSolver(mesh, br0) as s:
        x = np.zeros(s.N)
        r = s.rhs()
        assert s.cgsolve(x, r, ncgmax=5, epscg=1e-14) == 1
        assert s.last_info.ncg == 5


def test_device_pointer_solve_and_warm_guess(cuda):
    import torch
    mesh, br0 = _case(63, 91, 181)
    with Pot3dSolver(mesh, br0) as s:
        b = s.rhs()
        x = np.zeros(s.N)
        r = b.copy()
        s.cgsolve(x, r, epscg=1e-10)
        n_cold = s.last_info.ncg
        xt = torch.zeros(s.N, dtype=torch.float64, device=cuda)
        rt = torch.tensor(b, device=cuda)
        assert s.cgsolve_dev(xt, rt, epscg=1e-10) == 0
        assert np.array_equal(xt.cpu().numpy(), x)  # same arithmetic, same result
        # a guess close to the solution converges in fewer iterations
        x2 = x * (1 + 1e-4 * np.random.default_rng(1).standard_normal(s.N))
        r2 = b.copy()
        assert s.cgsolve(x2, r2, epscg=1e-10) == 0
        assert s.last_info.ncg < n_cold
        assert np.linalg.norm(x2 - x) <= 1e-6 * np.linalg.norm(x)


def test_kernel_timing_entry_point(cuda):
    mesh, br0 = _case(63, 91, 181)
    with Pot3dSolver(mesh, br0) as s:
        ms, by = s.time_kernels(5)
        assert np.all(ms > 0) and by[0] == 32.0 * s.N and by[1] == 48.0 * s.N


@pytest.mark.parametrize("dims,option", [((63, 91, 181), "ss"), ((37, 30, 26), "open")])
def test_fp32_refined_solve_parity(cuda, dims, option):
    """FP32 inner iterations with FP64 reliable updates reach the same
    solution as the FP64 oracle at epscg 1e-11: convergence is decided on the
    reference's epsn of the true FP64 residual."""
    mesh, br0 = _case(*dims, option=option)
    o = _oracle(mesh, br0, option=option)
    ref = o.cgsolve(np.zeros(o.N), o.rhs(), epscg=1e-11)
    phi_ref = o.finalize_phi(ref["x"])
    w_ref = o.energy(phi_ref)
    out = potfld(mesh, br0, option=option, precision="fp32_refined", epscg=1e-11)
    assert out["ierr"] == 0 and out["epsn"] < 1e-11
    assert out["n_refine"] >= 1
    rel = np.linalg.norm(out["phi"] - phi_ref) / np.linalg.norm(phi_ref)
    assert rel <= 1e-8, rel
    assert np.all(np.abs(out["energy"] - w_ref) <= 1e-9 * np.abs(w_ref))
    # the refined recurrence keeps the Krylov direction: few extra iterations
    assert out["ncg"] <= 1.5 * ref["ncg"] + 20, (out["ncg"], ref["ncg"])


def test_fp32_refined_true_residual_and_history(cuda):
    mesh, br0 = _case(63, 91, 181)
    out = potfld(mesh, br0, precision="fp32_refined", epscg=1e-9)
    assert out["ierr"] == 0
    # the returned r is the FP64 true residual b - A x of the returned x
    assert out["true_resid"] < 1e-7
    h = out["history"]
    assert len(h) == out["ncg"] + 1 and h[-1] < 1e-9
