"""The oracle against the reference's own test-suite outputs (CPU).

Pins: the mesh tables printed in testsuite/<case>/reference/pot3d.out, the
energies (7 decimals, as bin/pot3d_validation.sh compares), the iteration
count and the convergence history.  The PFSS case runs in full here; the
two larger cases run with POT3D_SLOW=1.
"""
import numpy as np
import pytest

import oracle as O
from conftest import CASES, load_case


def mesh_for(nml):
    return O.make_mesh(nml["nr"], nml["nt"], nml["np"], r0=nml["r0"], r1=nml["r1"], rfrac=nml["rfrac"],
                       drratio=nml["drratio"], nfrmesh=nml["nfrmesh"], tfrac=nml["tfrac"], dtratio=nml["dtratio"],
                       nftmesh=nml["nftmesh"], pfrac=nml["pfrac"], dpratio=nml["dpratio"], nfpmesh=nml["nfpmesh"],
                       phishift=nml["phishift"])


@pytest.mark.parametrize("case", CASES)
def test_mesh_tables(case):
    meta, _ = load_case(case)
    m = mesh_for(meta["namelist"])
    tabs = meta["reference"]["mesh_tables"]
    for lab, arr in (("r", m.r), ("t", m.t), ("p", m.p[:-1])):
        ref = np.array([v for _, v in tabs[lab]])
        assert ref.size == arr.size
        # pot3d.out prints f18.8
        assert np.max(np.abs(np.round(arr, 8) - ref)) <= 1.5e-8, lab


def _run_case(case):
    meta, z = load_case(case)
    nml = meta["namelist"]
    m = mesh_for(nml)
    br0 = O.readbr(m, z["tn"], z["pn"], np.asarray(z["data"], np.float64), nml["option"], nml["do_not_balance_flux"])
    out = O.potfld(m, br0, option=nml["option"], ifprec=nml["ifprec"], epscg=nml["epscg"], ncghist=nml["ncghist"])
    return meta["reference"], out


def _check(ref, out):
    w = out["energy"]
    for val, key in zip(w, ("wr", "wt", "wp")):
        assert round(val, 7) == round(ref["energy"][key], 7), key
        assert abs(val - ref["energy"][key]) <= 1e-9 * abs(ref["energy"][key])
    assert out["ncg"] == ref["iterations"]
    hist = dict(out["history"])
    for it, e in ref["history"]:
        assert abs(hist[it] - e) <= 1e-9 * e


def test_pfss_case_matches_reference():
    ref, out = _run_case("potential_field_source_surface")
    _check(ref, out)


@pytest.mark.slow
@pytest.mark.parametrize("case", CASES[1:])
def test_large_cases_match_reference(case):
    ref, out = _run_case(case)
    _check(ref, out)


def test_operator_is_symmetric_spd_small():
    m = O.make_mesh(6, 7, 9)
    br0 = np.zeros((7, 9), order="F")
    s = O.Solver(m, br0, "ss", 1)
    A = np.stack([s.ax(e) for e in np.eye(s.N)], axis=1)
    # The south-pole ghost couples the j=ntm1 ring through st(ntm1)=sin(pi)~1e-16.
    assert np.max(np.abs(A - A.T)) <= 1e-14 * np.max(np.abs(A))
    assert np.min(np.linalg.eigvalsh(0.5 * (A + A.T))) > 0


def test_coefficient_symmetry():
    m = O.make_mesh(7, 8, 10)
    s = O.Solver(m, np.zeros((8, 10), order="F"), "ss", 1)
    a = s.coef().reshape(7, 8, 6, 5)  # (coef, k, j, i) with nrm2=5, ntm2=6, npm2=8
    # a5(i) == a3(i+1), a6(j) == a2(j+1), a7(k) == a1(k+1)
    assert np.array_equal(a[4][:, :, :-1], a[2][:, :, 1:])
    assert np.array_equal(a[5][:, :-1, :], a[1][:, 1:, :])
    assert np.array_equal(a[6][:-1], a[0][1:])


@pytest.mark.parametrize("dims", [(8, 7, 9), (6, 9, 12), (9, 6, 7)])
def test_ilu0_only_changes_the_diagonal(dims):
    """For the 7-point pattern with np>=6 ILU(0) has no off-diagonal updates:
    the factor is the diagonal recurrence d_i = a_ii - sum_k (a_ik/d_k) a_ki."""
    nr, nt, np_ = dims
    m = O.make_mesh(nr, nt, np_)
    s = O.Solver(m, np.zeros((nt, np_), order="F"), "ss", 2)
    ia, ja, a = s.csr()
    f, icode = O.ilu0_csr(ia, ja, a)
    assert icode == 0
    N = ia.size - 1
    d = np.zeros(N, np.float32)
    for i in range(N):
        lo, hi = ia[i] - 1, ia[i + 1] - 1
        cols = ja[lo:hi] - 1
        for p in range(lo, hi):
            if cols[p - lo] > i:
                assert f[p] == a[p]  # U unchanged
        diag = lo + int(np.nonzero(cols == i)[0][0])
        di = np.float32(a[diag])
        for p in range(lo, diag):  # ascending columns
            k = cols[p - lo]
            lk = np.float32(a[p] / d[k])
            assert f[p] == lk
            klo, khi = ia[k] - 1, ia[k + 1] - 1
            q = klo + int(np.nonzero(ja[klo:khi] - 1 == i)[0][0])
            di = np.float32(di - np.float32(lk * a[q]))
        d[i] = di
        assert f[diag] == di
    dd, _ = s.ilu_diag()
    assert np.array_equal(dd, d)


def test_zero_rhs_returns_zero_solution():
    m = O.make_mesh(6, 7, 9)
    s = O.Solver(m, np.zeros((7, 9), order="F"), "ss", 1)
    out = s.cgsolve(np.ones(s.N), np.zeros(s.N))
    assert out["ierr"] == 0 and out["ncg"] == 0 and not out["x"].any()


def test_ncgmax_exceeded_sets_ierr():
    m = O.make_mesh(12, 13, 17)
    br0 = np.ones((13, 17), order="F")
    s = O.Solver(m, br0, "ss", 1)
    out = s.cgsolve(np.zeros(s.N), s.rhs(), ncgmax=3, epscg=1e-12)
    assert out["ierr"] == 1 and out["ncg"] == 3


def test_getb_restatement_and_energy_consistency():
    """orc_getb is src/pot3d.F90:6217-6231 (checked bit for bit against a
    numpy statement of the same formulas), and magnetic_energy, which
    evaluates B in place, equals the face-averaged energy of getb's fields."""
    m = O.make_mesh(11, 9, 14)
    rng = np.random.default_rng(3)
    s = O.Solver(m, np.zeros((9, 14), order="F"), "ss", 1)
    phi = s.finalize_phi(rng.standard_normal(s.N))
    br, bt, bp = s.getb(phi)
    dr, rh, dt, sth, dp = m.dr, m.rh, m.dt, m.sth, m.dp
    assert np.array_equal(br, (phi[1:] - phi[:-1]) / dr[:10, None, None])
    assert np.array_equal(bt, (phi[:, 1:] - phi[:, :-1]) / (rh[:, None, None] * dt[None, :8, None]))
    den = (rh[:, None] * sth[None, :])[:, :, None] * dp[None, None, :13]
    assert np.array_equal(bp, (phi[:, :, 1:] - phi[:, :, :-1]) / den)
    # energy over the interior with face averages (src/pot3d.F90:6279-6292)
    brav = 0.5 * (br[1:, 1:-1, 1:-1] + br[:-1, 1:-1, 1:-1])
    btav = 0.5 * (bt[1:-1, 1:, 1:-1] + bt[1:-1, :-1, 1:-1])
    bpav = 0.5 * (bp[1:-1, 1:-1, 1:] + bp[1:-1, 1:-1, :-1])
    dv = (rh[1:-1] ** 2 * m.drh[1:-1])[:, None, None] * (m.dth[1:-1] * sth[1:-1])[None, :, None] \
        * m.dph[None, None, 1:-1]
    w = [np.sum(0.5 * b * b * dv) for b in (brav, btav, bpav)]
    assert np.allclose(s.energy(phi), w, rtol=1e-12, atol=0)
