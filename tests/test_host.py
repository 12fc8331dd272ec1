"""Host-side pieces on CPU: meshes, br0, namelists, PSI HDF5 reader, and
the C-ABI library's exported symbols."""
import os
import re

import numpy as np
import pytest

import oracle as O
from conftest import CASES, GOLD, ROOT, load_case
from pot3d_b200 import _lib, host, namelist
from pot3d_b200.psi_io import PsiFormatError, read_psi

MESH_CONFIGS = [
    (55, 181, 361, {}),
    (101, 181, 361, dict(r0=2.5, r1=20.0, drratio=(40.0,), nfrmesh=5, tfrac=(0, 0.5, 1.0), dtratio=(0.5, 2.0),
                         nftmesh=5, nfpmesh=5)),
    (23, 17, 29, dict(pfrac=(0.2, 0.6), dpratio=(2.0, 0.5), nfpmesh=2, phishift=0.3)),
    (40, 30, 50, dict(pfrac=(0.0, 0.5), dpratio=(3.0, 0.3), rfrac=(0, 0.3, 1.0), drratio=(2.0, 4.0), nfrmesh=3)),
    (63, 91, 181, {}),
]


@pytest.mark.parametrize("nr,nt,np_,kw", MESH_CONFIGS)
def test_mesh_matches_oracle_bitwise(nr, nt, np_, kw):
    a = host.make_mesh(nr, nt, np_, **kw)
    b = O.make_mesh(nr, nt, np_, **kw)
    for f in O.MESH_FIELDS:
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


@pytest.mark.parametrize("case", CASES)
def test_br0_matches_oracle_on_testsuite_maps(case):
    meta, z = load_case(case)
    nml = meta["namelist"]
    m = host.mesh_from_namelist(nml)
    mo = O.make_mesh(nml["nr"], nml["nt"], nml["np"], r0=nml["r0"], r1=nml["r1"], rfrac=nml["rfrac"],
                     drratio=nml["drratio"], nfrmesh=nml["nfrmesh"], tfrac=nml["tfrac"], dtratio=nml["dtratio"],
                     nftmesh=nml["nftmesh"], pfrac=nml["pfrac"], dpratio=nml["dpratio"], nfpmesh=nml["nfpmesh"],
                     phishift=nml["phishift"])
    fi = np.asarray(z["data"], np.float64)
    a = host.br0_from_map(m, z["tn"], z["pn"], fi, nml["option"], nml["do_not_balance_flux"])
    b = O.readbr(mo, z["tn"], z["pn"], fi, nml["option"], nml["do_not_balance_flux"])
    assert np.array_equal(a, b)


def test_synthetic_br_properties():
    tn, pn, fi = host.synthetic_br(2, 40, 20, 361, 721)
    tn2, pn2, fi2 = host.synthetic_br(2, 40, 20, 361, 721)
    assert np.array_equal(fi, fi2)  # seeded
    w = np.sin(tn)[:, None] * np.ones((1, 720))
    assert abs((fi[:, :-1] * w).sum() / w.sum()) < 1e-12  # zero net flux
    assert 40 < np.abs(fi).max() < 120  # bipoles reach ~50 G over a 5 G background
    assert np.allclose(fi[:, 0], fi[:, -1], atol=1e-9)  # periodic in phi
    _, _, f3 = host.synthetic_br(3, 40, 20, 361, 721)
    assert not np.allclose(fi, f3)


def test_genmesh_errors_like_reference():
    with pytest.raises(ValueError):
        host.genmesh(1, 0.0, 1.0, (0.0,), (1.0,))
    with pytest.raises(ValueError):
        host.genmesh(10, 1.0, 0.0, (0.0,), (1.0,))
    with pytest.raises(ValueError):  # non-periodic FRAC must end at 1
        host.genmesh(10, 0.0, 1.0, (0.0, 0.5), (2.0,))
    with pytest.raises(ValueError):  # periodic FRAC must not hold both 0 and 1
        host.genmesh(10, 0.0, 1.0, (0.0, 1.0), (2.0, 2.0), periodic=True)


@pytest.mark.parametrize("case", CASES)
def test_namelist_fixture_roundtrip(case):
    meta, _ = load_case(case)
    v = meta["namelist"]
    assert v["nr"] > 2 and v["option"] in ("ss", "open", "potential")
    assert v["ifprec"] == 1 and v["epscg"] == 1e-9


def test_namelist_parser_defaults_and_errors():
    txt = """ &topology
  nr=63
  nt=91 ! comment
  np=181
 /
 &inputvars
  option='ss'
  rfrac=0.0,1.0
  drratio=2.5
  do_not_balance_flux=.true.
  epscg=1.d-11
 /
"""
    n = namelist.parse(txt)
    assert (n.nr, n.nt, n.np) == (63, 91, 181)
    assert n.rfrac[:3] == [0.0, 1.0, 0.0] and n.drratio[0] == 2.5
    assert n.do_not_balance_flux is True and n.epscg == 1e-11
    assert n.ifprec == 1 and n.ncghist == 100 and n.r1 == 30.0  # module defaults
    assert n.pm_r1 == -1.0
    with pytest.raises(namelist.NamelistError):
        namelist.parse(txt.replace("epscg", "bogus_key"))


def test_psi_reader_on_fixture_shapes():
    # The fixture npz files were produced by read_psi from the reference's
    # shipped maps; the scales there are monotone and span [0,pi]x[0,2pi].
    for case in CASES:
        _, z = load_case(case)
        assert z["data"].shape == (z["tn"].size, z["pn"].size)
        assert np.all(np.diff(z["tn"]) > 0) and np.all(np.diff(z["pn"]) > 0)


def test_psi_reader_rejects_garbage(tmp_path):
    p = tmp_path / "bad.h5"
    p.write_bytes(b"not an hdf5 file at all")
    with pytest.raises(PsiFormatError):
        read_psi(str(p))
    p.write_bytes(b"\x89HDF\r\n\x1a\n" + b"\x00" * 20)
    with pytest.raises(PsiFormatError):
        read_psi(str(p))


def _declared_symbols():
    syms = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(\w+)\s*\(", txt, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "return", "sizeof") and not name.startswith("POT3D"):
                syms.add(name)
    return syms


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    syms = _declared_symbols()
    assert {"load_external_lu_solver", "external_lu_solver", "pot3d_gpu_cgsolve"} <= syms
    missing = [s for s in sorted(syms) if not hasattr(L, s)]
    assert not missing, missing


def test_batch_specs_cover_the_uneven_grid_law():
    from pot3d_b200.batch import NP, NR, NT, batch_specs
    s = batch_specs(48, 0)
    assert len(s) == 48 and s == batch_specs(48, 0)
    assert {x[0] for x in s} <= set(NR) and {x[1] for x in s} <= set(NT) and {x[2] for x in s} <= set(NP)
    assert len({x[:3] for x in s}) > 4  # uneven
    assert all(2.0 <= x[3] <= 3.0 for x in s)
    assert len({x[4] for x in s}) == 48  # own Br seed per case


@pytest.mark.parametrize("args", [(1, 15, 4, 91, 181), (2, 40, 20, 361, 721), (7, 5, 0, 13, 17),
                                  (100, 40, 20, 91, 181)])
def test_oracle_generator_matches_product_bitwise(args):
    """The oracle's restatement of the seeded Br generator gives the product
    generator's maps bit for bit, so the CPU reference arm can build the
    workloads without the product library."""
    a = O.synthetic_br(*args)
    b = host.synthetic_br(*args)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_oracle_builds_the_bench_workload_bitwise():
    w = host.WORKLOADS["pfss_63x91x181"]
    m1, b1 = O.pfss_case(w["nr"], w["nt"], w["np"], w["lmax"], w["nbip"], w["seed"])
    m2, b2 = host.pfss_case(w["nr"], w["nt"], w["np"], w["lmax"], w["nbip"], w["seed"])
    assert np.array_equal(b1, b2)
    for f in O.MESH_FIELDS:
        assert np.array_equal(getattr(m1, f), getattr(m2, f))
