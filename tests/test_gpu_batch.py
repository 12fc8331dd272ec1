"""Batched PCG over uneven grids against single-case solves.

With the default planes per block every case runs the same tiles and the same
reduction order as its single-case solve, so iteration counts and solutions
must agree bit for bit; a tuned planes-per-block changes only the summation
order of the reductions (iterations within 1, solutions to 1e-9 relative).
"""
import numpy as np
import pytest

from pot3d_b200 import host
from pot3d_b200.host import PM_R1
from pot3d_b200.solver import BatchSolver, Pot3dSolver

pytestmark = pytest.mark.gpu

DIMS = [(33, 41, 65, 2.0), (25, 31, 48, 2.7), (41, 37, 73, 3.0), (20, 13, 11, 2.3)]


def _cases():
    out = []
    for q, (nr, nt, np_, r1) in enumerate(DIMS):
        mesh = host.make_mesh(nr, nt, np_, r1=r1)
        tn, pn, fi = host.synthetic_br(100 + q, 15, 4, nt, np_)
        out.append((mesh, host.br0_from_map(mesh, tn, pn, fi)))
    return out


def _single(mesh, br0, epscg, ifprec=1):
    with Pot3dSolver(mesh, br0, ifprec=ifprec) as s:
        x = np.zeros(s.N)
        r = s.rhs()
        ierr = s.cgsolve(x, r, epscg=epscg)
        return ierr, s.last_info.ncg, x


def test_batch_matches_single_solves_bitwise(cuda):
    cases = _cases()
    with BatchSolver([c[0] for c in cases], [c[1] for c in cases], [PM_R1["ss"]] * len(cases)) as b:
        ierr = b.solve(epscg=1e-10)
        assert ierr == [0] * len(cases)
        ncgs = [i.ncg for i in b.infos]
        assert len(set(ncgs)) > 1  # the cases stop at different iterations
        for q, (mesh, br0) in enumerate(cases):
            e1, n1, x1 = _single(mesh, br0, 1e-10)
            assert e1 == 0 and n1 == ncgs[q]
            assert np.array_equal(b.solution(q), x1)
        # a second solve on the same batch (graph reused) repeats the first
        x0 = b.solution(0)
        assert b.solve(epscg=1e-10) == [0] * len(cases)
        assert [i.ncg for i in b.infos] == ncgs
        assert np.array_equal(b.solution(0), x0)


def test_batch_tuned_planes_per_block(cuda):
    cases = _cases()
    with BatchSolver([c[0] for c in cases], [c[1] for c in cases], [PM_R1["ss"]] * len(cases)) as b:
        best, times = b.tune(candidates=(8, 16, 32), iters=4)
        assert best in (8, 16, 32) and all(t > 0 for t in times.values())
        assert b.solve(epscg=1e-10) == [0] * len(cases)


@pytest.mark.parametrize("precision", ["fp64", "fp32_refined"])
def test_batch_two_parameter_tuner(cuda, precision):
    """Stencil and update planes per block tuned together (the update's
    finest chunking, 8 planes, included): every pair runs, and the batch
    then solves to the single-case solutions."""
    cases = _cases()
    with BatchSolver([c[0] for c in cases], [c[1] for c in cases], [PM_R1["ss"]] * len(cases), ifprec=2,
                     precision=precision) as b:
        (bt, btu), times = b.tune2(candidates=(8, 32), update_candidates=(8, 64), iters=3)
        assert bt in (8, 32) and btu in (8, 64) and len(times) == 4 and all(t > 0 for t in times.values())
        assert b.solve(epscg=1e-10, ncgmax=20000) == [0] * len(cases)
        for q, (mesh, br0) in enumerate(cases):
            e1, n1, x1 = _single(mesh, br0, 1e-10, ifprec=2)
            assert np.linalg.norm(b.solution(q) - x1) <= 1e-8 * np.linalg.norm(x1)
            if precision == "fp64":
                assert abs(b.infos[q].ncg - n1) <= 1


def test_batch_zero_rhs_case(cuda):
    cases = _cases()[:2]
    cases[1] = (cases[1][0], np.zeros_like(cases[1][1]))
    with BatchSolver([c[0] for c in cases], [c[1] for c in cases], [PM_R1["ss"]] * 2) as b:
        assert b.solve(epscg=1e-10) == [0, 0]
        assert b.infos[1].ncg == 0
        assert not b.solution(1).any()
        e1, n1, x1 = _single(*cases[0], 1e-10)
        assert b.infos[0].ncg == n1 and np.array_equal(b.solution(0), x1)


def test_batch_rejects_bad_arguments(cuda):
    from pot3d_b200._lib import Pot3dError
    mesh, br0 = _cases()[0]
    with pytest.raises(Pot3dError):
        BatchSolver([mesh], [br0], [1.0], tk=3)
    with BatchSolver([mesh], [br0], [1.0]) as b:
        with pytest.raises(Pot3dError):
            b.tune(candidates=(4,))


def test_ilu_batch_matches_single_ilu_solves_bitwise(cuda):
    """ILU(0) batch: the stencil, update and r.z run the single-case bodies on
    the same tiles and the batched sweeps compute every value as the
    single-case sweeps do, so iterations and solutions are bit-identical."""
    cases = _cases()
    with BatchSolver([c[0] for c in cases], [c[1] for c in cases], [PM_R1["ss"]] * len(cases), ifprec=2) as b:
        for rep in range(2):  # the sweeps' tickets and tags carry over between solves
            ierr = b.solve(epscg=1e-10)
            assert ierr == [0] * len(cases)
            ncgs = [i.ncg for i in b.infos]
            for q, (mesh, br0) in enumerate(cases):
                e1, n1, x1 = _single(mesh, br0, 1e-10, ifprec=2)
                assert e1 == 0 and n1 == ncgs[q]
                assert np.array_equal(b.solution(q), x1)
        diag = BatchSolver([c[0] for c in cases], [c[1] for c in cases], [PM_R1["ss"]] * len(cases))
        diag.solve(epscg=1e-10)
        assert all(i.ncg < j.ncg for i, j in zip(b.infos, diag.infos))
        diag.close()


def test_batch_rejects_bad_preconditioner(cuda):
    from pot3d_b200._lib import Pot3dError
    mesh, br0 = _cases()[0]
    with pytest.raises(Pot3dError):
        BatchSolver([mesh], [br0], [1.0], ifprec=3)


@pytest.mark.parametrize("ifprec", [1, 2])
def test_batch_matches_the_oracle(cuda, ifprec):
    """Every case of an uneven batch (own grid, map and source-surface
    radius) solved to 1e-11 by the batched kernels lands on the oracle's
    solution of that case (the reference's CPU PCG with the same
    preconditioner): relative L2 <= 1e-8 on the packed solution."""
    import oracle as O
    cases = _cases()
    with BatchSolver([c[0] for c in cases], [c[1] for c in cases], [PM_R1["ss"]] * len(cases), ifprec=ifprec) as b:
        assert b.solve(epscg=1e-11) == [0] * len(cases)
        for q, (mesh, br0) in enumerate(cases):
            mo = O.Mesh(mesh.nr, mesh.nt, mesh.np, *[getattr(mesh, f) for f in O.MESH_FIELDS])
            o = O.Solver(mo, br0, "ss", ifprec)
            ref = o.cgsolve(np.zeros(o.N), o.rhs(), epscg=1e-11)
            x = b.solution(q)
            assert np.linalg.norm(x - ref["x"]) <= 1e-8 * np.linalg.norm(ref["x"]), q
            assert abs(b.infos[q].ncg - ref["ncg"]) <= max(2, ref["ncg"] // 50), (q, b.infos[q].ncg, ref["ncg"])


@pytest.mark.parametrize("ifprec", [1, 2])
def test_refined_batch_matches_the_oracle(cuda, ifprec):
    """FP32-inner / FP64-refined batch (per-case reliable updates and
    convergence on each case's FP64 residual): every case lands on the
    oracle's FP64 solution at 1e-11, with iteration counts close to the
    FP64 ones."""
    import oracle as O
    cases = _cases()
    with BatchSolver([c[0] for c in cases], [c[1] for c in cases], [PM_R1["ss"]] * len(cases), ifprec=ifprec,
                     precision="fp32_refined") as b:
        assert b.solve(epscg=1e-11, ncgmax=20000) == [0] * len(cases)
        for q, (mesh, br0) in enumerate(cases):
            mo = O.Mesh(mesh.nr, mesh.nt, mesh.np, *[getattr(mesh, f) for f in O.MESH_FIELDS])
            o = O.Solver(mo, br0, "ss", ifprec)
            ref = o.cgsolve(np.zeros(o.N), o.rhs(), epscg=1e-11)
            x = b.solution(q)
            assert np.linalg.norm(x - ref["x"]) <= 1e-8 * np.linalg.norm(ref["x"]), q
            assert b.infos[q].n_refine >= 1
            assert b.infos[q].ncg <= 1.2 * ref["ncg"] + 16, (q, b.infos[q].ncg, ref["ncg"])
        # from per-case guesses near the solutions: fewer iterations, same solutions
        sols = [b.solution(q) for q in range(len(cases))]
        ncg0 = [i.ncg for i in b.infos]
        rng = np.random.default_rng(5)
        for q, x in enumerate(sols):
            b.set_guess(q, x * (1.0 + 1e-2 * rng.standard_normal(x.size)))
        assert b.solve(epscg=1e-11, ncgmax=20000) == [0] * len(cases)
        for q, x in enumerate(sols):
            assert np.linalg.norm(b.solution(q) - x) <= 1e-8 * np.linalg.norm(x)
            assert b.infos[q].ncg < ncg0[q]


def test_batch_guess_fp64_and_reset(cuda):
    cases = _cases()
    with BatchSolver([c[0] for c in cases], [c[1] for c in cases], [PM_R1["ss"]] * len(cases), ifprec=2) as b:
        assert b.solve(epscg=1e-10) == [0] * len(cases)
        ncg0 = [i.ncg for i in b.infos]
        x0 = b.solution(1)
        b.set_guess(1, x0)  # the converged solution as the guess: almost nothing to do
        assert b.solve(epscg=1e-10) == [0] * len(cases)
        assert b.infos[1].ncg < ncg0[1] // 2
        assert np.linalg.norm(b.solution(1) - x0) <= 1e-9 * np.linalg.norm(x0)
        b.set_guess(1, None)
        assert b.solve(epscg=1e-10) == [0] * len(cases)
        assert [i.ncg for i in b.infos] == ncg0
        with pytest.raises(ValueError):
            b.set_guess(0, np.zeros(3))
