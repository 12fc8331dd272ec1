"""GPU parity of the FP32-inner / FP64-refined PCG with both preconditioners,
and of the FP64 ILU(0) solve on the 63x91x181 PFSS workload, against the
oracle (the CPU restatement of the reference's cgsolve with ifprec=1 and 2).

Every solve here runs to epscg 1e-11 and is compared with the oracle's solve
of the same inputs: phi relative L2 <= 1e-8 and energies <= 1e-9 relative
(the tolerances of the reference comparison).  The refined solve decides
convergence on the reference's epsn of the FP64 residual b - A x, so it must
land on the same solution; its inner FP32 recurrence may take a few more
iterations than FP64 PCG.
"""
import numpy as np
import pytest

import oracle as O
from pot3d_b200 import host
from pot3d_b200.solver import Pot3dSolver, potfld

pytestmark = pytest.mark.gpu

EPS = 1e-11
NCGMAX = 20000  # a failing solve ends in seconds, not at the default cap


def _case(nr, nt, np_, seed=3, option="ss", lmax=15, nbip=4):
    mesh = host.make_mesh(nr, nt, np_)
    tn, pn, fi = host.synthetic_br(seed, lmax, nbip, nt, np_)
    return mesh, host.br0_from_map(mesh, tn, pn, fi, option=option)


_REF = {}


def _oracle_solution(key, mesh, br0, option, ifprec):
    """Oracle solve at 1e-11 (phi, energies, iterations), cached per module."""
    if key not in _REF:
        mo = O.Mesh(mesh.nr, mesh.nt, mesh.np, *[getattr(mesh, f) for f in O.MESH_FIELDS])
        o = O.Solver(mo, br0, option, ifprec)
        ref = o.cgsolve(np.zeros(o.N), o.rhs(), epscg=EPS)
        phi = o.finalize_phi(ref["x"])
        _REF[key] = dict(x=ref["x"], phi=phi, w=o.energy(phi), ncg=ref["ncg"])
    return _REF[key]


def _check(out, ref):
    assert out["ierr"] == 0 and out["epsn"] < EPS
    rel = np.linalg.norm(out["phi"] - ref["phi"]) / np.linalg.norm(ref["phi"])
    assert rel <= 1e-8, rel
    assert np.all(np.abs(out["energy"] - ref["w"]) <= 1e-9 * np.abs(ref["w"])), (out["energy"], ref["w"])
    return rel


C1 = (63, 91, 181)


def _c1():
    w = host.WORKLOADS["pfss_63x91x181"]
    return host.pfss_case(w["nr"], w["nt"], w["np"], w["lmax"], w["nbip"], w["seed"])


def test_c1_ilu_fp64_matches_oracle():
    """FP64 PCG with ILU(0) on the 63x91x181 PFSS workload (seed 1), from
    zero, against the oracle's ifprec=2 solve."""
    mesh, br0 = _c1()
    ref = _oracle_solution(("c1", 2), mesh, br0, "ss", 2)
    out = potfld(mesh, br0, ifprec=2, epscg=EPS, ncgmax=NCGMAX)
    _check(out, ref)
    assert abs(out["ncg"] - ref["ncg"]) <= max(2, ref["ncg"] // 50), (out["ncg"], ref["ncg"])


@pytest.mark.parametrize("ifprec", [1, 2])
def test_c1_refined_matches_oracle(ifprec):
    """FP32-inner / FP64-refined PCG on the 63x91x181 workload matches the
    oracle's FP64 solve, from zero and from a perturbed guess."""
    mesh, br0 = _c1()
    ref = _oracle_solution(("c1", ifprec), mesh, br0, "ss", ifprec)
    out = potfld(mesh, br0, ifprec=ifprec, precision="fp32_refined", epscg=EPS, ncgmax=NCGMAX)
    _check(out, ref)
    assert out["n_refine"] >= 1
    # FP32 storage of p, q, r costs few iterations: the products are FP64
    assert out["ncg"] <= 1.2 * ref["ncg"] + 10, (out["ncg"], ref["ncg"])
    # a guess near the solution (1% noise) converges to the same phi in fewer iterations
    rng = np.random.default_rng(11)
    x0 = ref["x"] * (1.0 + 1e-2 * rng.standard_normal(ref["x"].size))
    out2 = potfld(mesh, br0, ifprec=ifprec, precision="fp32_refined", epscg=EPS, x0=x0, ncgmax=NCGMAX)
    _check(out2, ref)
    assert out2["ncg"] < out["ncg"]


def test_c1_ilu_fp64_from_perturbed_guess():
    mesh, br0 = _c1()
    ref = _oracle_solution(("c1", 2), mesh, br0, "ss", 2)
    rng = np.random.default_rng(12)
    x0 = ref["x"] * (1.0 + 1e-2 * rng.standard_normal(ref["x"].size))
    out = potfld(mesh, br0, ifprec=2, epscg=EPS, x0=x0, ncgmax=NCGMAX)
    _check(out, ref)


@pytest.mark.parametrize("dims,option", [((37, 30, 26), "ss"), ((20, 13, 11), "open"), ((9, 7, 8), "ss")])
def test_refined_ilu_small_grids(dims, option):
    """Partial tiles, one tile and a single-tile wavefront."""
    mesh, br0 = _case(*dims, option=option)
    ref = _oracle_solution((dims, option, 2), mesh, br0, option, 2)
    out = potfld(mesh, br0, option=option, ifprec=2, precision="fp32_refined", epscg=EPS, ncgmax=NCGMAX)
    _check(out, ref)


@pytest.mark.parametrize("ifprec", [1, 2])
def test_refined_stagnation_switches_to_fp64(ifprec):
    """With a stagnation test no update can pass (stall_drop tiny), the
    second reliable update hands the solve to FP64 PCG from the current x;
    the result is still the oracle's solution."""
    mesh, br0 = _case(37, 30, 26)
    ref = _oracle_solution(((37, 30, 26), "ss", ifprec), mesh, br0, "ss", ifprec)
    with Pot3dSolver(mesh, br0, ifprec=ifprec, precision="fp32_refined") as s:
        s.set_refine(refine_ratio=1e-2, stall_drop=1e-300, stall_limit=2)
        b = s.rhs()
        x = np.zeros(s.N)
        r = b.copy()
        assert s.cgsolve(x, r, epscg=EPS, ncgmax=NCGMAX) == 0
        n_ref, fb = s.refine_info()
        assert n_ref == 2 and fb > 0, (n_ref, fb)
        assert s.last_info.epsn < EPS
        phi = s.finalize_phi(x)
        w = s.energy(phi)
    rel = np.linalg.norm(phi - ref["phi"]) / np.linalg.norm(ref["phi"])
    assert rel <= 1e-8, rel
    assert np.all(np.abs(w - ref["w"]) <= 1e-9 * np.abs(ref["w"]))


def test_refined_solver_reuse_and_ncgmax():
    """Repeated refined solves on one handle give the same result; an ncgmax
    below the need returns ierr = 1 with a finite epsn."""
    mesh, br0 = _case(37, 30, 26)
    with Pot3dSolver(mesh, br0, ifprec=2, precision="fp32_refined") as s:
        b = s.rhs()
        xs = []
        for _ in range(2):
            x = np.zeros(s.N)
            r = b.copy()
            assert s.cgsolve(x, r, epscg=EPS, ncgmax=NCGMAX) == 0
            xs.append(x)
        assert np.array_equal(xs[0], xs[1])
        x = np.zeros(s.N)
        r = b.copy()
        assert s.cgsolve(x, r, ncgmax=5, epscg=EPS) == 1
        assert np.isfinite(s.last_info.epsn) and s.last_info.epsn > EPS
    with pytest.raises(Exception):
        with Pot3dSolver(mesh, br0, ifprec=2, precision="fp32_refined") as s:
            s.set_refine(refine_ratio=2.0)
