"""The one-solve driver (pot3d_b200.run) on the GPU.

* The reference's PFSS test-suite case, from a pot3d.dat and a PSI HDF5 Br
  map written to a run directory: the printed energies round to the
  reference's pot3d.out values at 7 decimals (bin/pot3d_validation.sh), the
  iteration count is within 1% of the reference's, and the written B files
  reproduce the printed energies.
* The validation run (tilted dipole, src/pot3d.F90:3978-4131): the same
  errors against the analytic field as the oracle's solve, and the
  discretisation error falls with the mesh (second order for br and bt;
  first order for bp, whose analytic values the reference evaluates with
  the half-mesh sin(ph)).
"""
import os

import numpy as np
import pytest

import oracle as O
from conftest import load_case
from pot3d_b200 import host
from pot3d_b200.psi_io import read_psi, write_psi
from pot3d_b200.run import _energy_lines, run

pytestmark = pytest.mark.gpu

_ANGLE = 0.7853981633974483


def _fmt(v):
    if isinstance(v, bool):
        return ".true." if v else ".false."
    if isinstance(v, str):
        return f"'{v}'"
    if isinstance(v, (list, tuple)):
        return ",".join(_fmt(x) for x in v)
    return repr(v)


def _write_dat(path, values):
    topo = {k: values[k] for k in ("nr", "nt", "np")}
    rest = {k: v for k, v in values.items() if k not in topo}
    with open(path, "w") as fh:
        fh.write(" &topology\n" + "".join(f"  {k}={_fmt(v)}\n" for k, v in topo.items()) + " /\n")
        fh.write(" &inputvars\n" + "".join(f"  {k}={_fmt(v)}\n" for k, v in rest.items()) + " /\n")


def _energy(br, bt, bp, m):
    """magnetic_energy (src/pot3d.F90:6279-6292) from stored B fields."""
    brav = 0.5 * (br[1:, 1:-1, 1:-1] + br[:-1, 1:-1, 1:-1])
    btav = 0.5 * (bt[1:-1, 1:, 1:-1] + bt[1:-1, :-1, 1:-1])
    bpav = 0.5 * (bp[1:-1, 1:-1, 1:] + bp[1:-1, 1:-1, :-1])
    dv = (m.rh[1:-1] ** 2 * m.drh[1:-1])[:, None, None] * (m.dth[1:-1] * m.sth[1:-1])[None, :, None] \
        * m.dph[None, None, 1:-1]
    return np.array([np.sum(0.5 * b * b * dv) for b in (brav, btav, bpav)])


@pytest.mark.parametrize("ifprec", [None, 2])
def test_driver_pfss_testsuite_case(cuda, tmp_path, ifprec):
    """ifprec None: the namelist's diagonal preconditioner.  ifprec 2:
    ILU(0), whose converged energies also round to the reference's (the
    oracle's ILU(0) solve takes 398 iterations here)."""
    meta, z = load_case("potential_field_source_surface")
    nml = dict(meta["namelist"])
    data = np.asarray(z["data"])
    write_psi(tmp_path / "br_input.h5", data, [z["tn"], z["pn"]], hdf32=data.dtype == np.float32)
    nml.update(br0file="br_input.h5", brfile="br.h5", btfile="bt.h5", bpfile="bp.h5", phifile="",
               br_photo_file="br_photo.h5", br_photo_original_file="")
    _write_dat(tmp_path / "pot3d.dat", nml)
    res = run(str(tmp_path / "pot3d.dat"), ifprec=ifprec, quiet=True)
    ref = meta["reference"]
    for val, key in zip(res["energy"], ("wr", "wt", "wp")):
        assert round(val, 7) == round(ref["energy"][key], 7), key
    if ifprec is None:
        assert abs(res["ncg"] - ref["iterations"]) <= max(3, ref["iterations"] // 100)
    else:
        assert abs(res["ncg"] - 398) <= 8
    assert not os.path.exists(tmp_path / "phi.h5")
    m = host.mesh_from_namelist(nml)
    br, bt, bp = (read_psi(tmp_path / f).data for f in ("br.h5", "bt.h5", "bp.h5"))
    assert br.shape == (m.nr - 1, m.nt, m.np) and bt.shape == (m.nr, m.nt - 1, m.np)
    assert bp.shape == (m.nr, m.nt, m.np - 1)
    assert np.allclose(_energy(br, bt, bp, m), res["energy"], rtol=1e-12, atol=0)
    photo = read_psi(tmp_path / "br_photo.h5")
    assert photo.data.shape == (m.nt, m.np) and np.allclose(photo.scales[0], m.th)
    out = (tmp_path / "pot3d.out").read_text().splitlines()
    assert out[-4:] == _energy_lines(res["energy"])
    assert "### The CG solver has converged." in " ".join(out)


def _validation_dat(path, dims, ifprec=1):
    nr, nt, np_ = dims
    _write_dat(path, dict(nr=nr, nt=nt, np=np_, option="ss", validation_run=True, r0=1.0, r1=2.5,
                          rfrac=[0.0, 1.0], drratio=[2.5], ifprec=ifprec, epscg=1e-11, ncghist=0,
                          dipole_angle=_ANGLE))


def test_driver_validation_run_matches_oracle(cuda, tmp_path):
    dims = (22, 41, 81)
    _validation_dat(tmp_path / "pot3d.dat", dims)
    res = run(str(tmp_path / "pot3d.dat"), quiet=True)
    for f in ("phi_exact", "br_exact", "bt_exact", "bp_exact", "brfile", "btfile", "bpfile", "phifile"):
        assert os.path.exists(res["files"][f]), f
    # the same solve on the oracle
    m = host.make_mesh(*dims, r1=2.5)
    mo = O.Mesh(m.nr, m.nt, m.np, *[getattr(m, f) for f in O.MESH_FIELDS])
    b0, b1 = host.validation_br(m, _ANGLE, 1.0, 2.5)
    o = O.Solver(mo, b0, "ss", 1, br1=b1)
    ref = o.cgsolve(np.zeros(o.N), o.rhs(), ncgmax=100000, epscg=1e-11)
    phi = o.finalize_phi(ref["x"])
    w_ref = o.energy(phi)
    assert np.all(np.abs(res["energy"] - w_ref) <= 1e-9 * np.abs(w_ref))
    assert abs(res["ncg"] - ref["ncg"]) <= max(3, ref["ncg"] // 50)
    _, brx, btx, bpx = host.validation_exact(m, _ANGLE)
    sl = (slice(1, -1),) * 3
    for f, got, ex in zip(("br", "bt", "bp"), o.getb(phi), (brx, btx, bpx)):
        e_ref = np.linalg.norm((got - ex)[sl]) / np.linalg.norm(ex[sl])
        assert abs(res["validation_rel_l2"][f] - e_ref) <= 1e-6 * e_ref, f


@pytest.mark.parametrize("ifprec", [1, 2])
def test_driver_validation_run_converges_with_the_mesh(cuda, tmp_path, ifprec):
    errs = []
    for dims in ((22, 41, 81), (42, 81, 161)):
        d = tmp_path / f"{dims[0]}"
        d.mkdir()
        _validation_dat(d / "pot3d.dat", dims, ifprec=ifprec)
        errs.append(run(str(d / "pot3d.dat"), quiet=True)["validation_rel_l2"])
    assert errs[1]["br"] < errs[0]["br"] / 3.5
    assert errs[1]["bt"] < errs[0]["bt"] / 3.5
    assert errs[1]["bp"] < errs[0]["bp"] / 1.8
    assert errs[1]["br"] < 1e-4 and errs[1]["bt"] < 1e-3 and errs[1]["bp"] < 0.03
