"""Host pieces of the one-solve driver on CPU: the PSI HDF5 writer, output
file names, the printed lines, and the validation-run boundary fields.
(The driver's GPU runs are in test_gpu_run.py.)"""
import numpy as np
import pytest

from conftest import load_case
from pot3d_b200 import host, namelist
from pot3d_b200.psi_io import read_psi, write_psi
from pot3d_b200.run import _energy_lines, _history_lines, field_scales, output_names


@pytest.mark.parametrize("shape", [(7,), (5, 9), (4, 6, 3)])
@pytest.mark.parametrize("hdf32", [False, True])
def test_write_psi_round_trip(tmp_path, shape, hdf32):
    rng = np.random.default_rng(len(shape))
    data = rng.standard_normal(shape)
    scales = [np.linspace(0.0, 1.0, n) for n in shape]
    p = tmp_path / "f.h5"
    write_psi(p, data, scales, hdf32=hdf32)
    d = read_psi(p)
    dt = np.float32 if hdf32 else np.float64
    assert d.dtype == np.dtype(dt)
    assert d.data.shape == shape
    assert np.array_equal(d.data, data.astype(dt))
    for s, ref in zip(d.scales, scales):
        assert np.array_equal(s, ref.astype(dt).astype(np.float64))


def test_write_psi_layout(tmp_path):
    """Members in the order rdh5 reads them (Data first, then dim1..dimN),
    each scale carrying CLASS = "DIMENSION_SCALE" as h5DSis_scale_f
    requires, and a file that ends where the superblock says."""
    p = tmp_path / "f.h5"
    write_psi(p, np.ones((3, 4)), [np.arange(3.0), np.arange(4.0)])
    buf = p.read_bytes()
    assert buf[:8] == b"\x89HDF\r\n\x1a\n"
    assert int.from_bytes(buf[40:48], "little") == len(buf)
    assert buf.count(b"CLASS\x00") == 2
    assert buf.count(b"DIMENSION_SCALE\x00") == 2
    heap = buf.index(b"HEAP")
    seg = int.from_bytes(buf[heap + 24:heap + 32], "little")
    assert buf[seg:seg + 32] == b"\x00" * 8 + b"Data\x00\x00\x00\x00dim1\x00\x00\x00\x00dim2\x00\x00\x00\x00"
    # one free block closes the heap's free list (next = 1, size 16)
    free = int.from_bytes(buf[heap + 16:heap + 24], "little")
    assert int.from_bytes(buf[seg + free:seg + free + 8], "little") == 1


def test_write_psi_rejects_bad_input(tmp_path):
    with pytest.raises(ValueError):
        write_psi(tmp_path / "a.h5", np.ones((2, 2, 2, 2)))
    with pytest.raises(ValueError):
        write_psi(tmp_path / "b.h5", np.ones((2, 3)), [np.arange(2.0)])
    with pytest.raises(ValueError):
        write_psi(tmp_path / "c.h5", np.ones((2, 3)), [np.arange(2.0), np.arange(4.0)])


def test_write_psi_no_scales(tmp_path):
    p = tmp_path / "f.h5"
    write_psi(p, np.arange(12.0).reshape(3, 4))
    d = read_psi(p)
    assert not d.has_scales
    assert np.array_equal(d.data, np.arange(12.0).reshape(3, 4))


def test_output_names():
    v = namelist.parse("&topology nr=5 nt=6 np=7 /\n&inputvars phifile='' brfile='b.h5' /").values
    n = output_names(v)
    assert n["phifile"] == "" and n["brfile"] == "b.h5"
    assert n["btfile"] == "bt.h5" and n["bpfile"] == "bp.h5" and n["br_photo_file"] == "br_photo.h5"
    assert n["outfile"] == "pot3d.out"
    v = namelist.parse("&topology nr=5 nt=6 np=7 /\n&inputvars validation_run=.true. phifile='' /").values
    n = output_names(v)
    assert (n["phifile"], n["brfile"], n["btfile"], n["bpfile"]) == ("phi_solved.h5", "br_solved.h5",
                                                                    "bt_solved.h5", "bp_solved.h5")


def test_energy_lines_reproduce_reference_text():
    meta, _ = load_case("potential_field_source_surface")
    e = meta["reference"]["energy"]
    lines = _energy_lines([e["wr"], e["wt"], e["wp"]])
    assert lines[:3] == meta["reference"]["energy_text"]


def test_history_lines_format():
    meta, _ = load_case("potential_field_source_surface")
    hist = np.full(meta["reference"]["iterations"] + 1, 0.5)
    for it, e in meta["reference"]["history"]:
        hist[it] = e
    hist[-1] = 9.903437008397958e-10
    lines = _history_lines(hist, 100, 1e-9)
    assert lines[1] == " ### Convergence information:"
    assert lines[2] == " Iteration:        0   Residual:   9.999999999999994E-01"
    assert lines[3] == " Iteration:      100   Residual:   5.171368006251082E-02"
    assert lines[-2] == " ### The CG solver has converged."
    assert lines[-1] == " Iteration:     2995   Residual:   9.903437008397958E-10"
    assert _history_lines(hist, 0, 1e-9) == []


def test_validation_boundary_fields():
    """set_validation_flux: periodic in phi, pole rows from the m=0
    average, and the dipole's 1/r^3 scaling between r0 and r1."""
    m = host.make_mesh(12, 21, 41, r1=2.5)
    b0, b1 = host.validation_br(m, 0.7853981633974483, 1.0, 2.5)
    assert b0.shape == (21, 41) and b1.shape == (21, 41)
    assert np.array_equal(b0[:, 0], b0[:, -2]) and np.array_equal(b0[:, -1], b0[:, 1])
    w = m.dph[1:-1] / (2 * np.pi)
    assert np.allclose(0.5 * (b0[0] + b0[1]), np.sum(b0[1, 1:-1] * w), rtol=0, atol=1e-14)
    assert np.allclose(b1[1:-1, 1:-1] * 2.5 ** 3, b0[1:-1, 1:-1], rtol=1e-13)
    x, br, bt, bp = host.validation_exact(m, 0.7853981633974483)
    assert x.size == m.N
    assert br.shape == (11, 21, 41) and bt.shape == (12, 20, 41) and bp.shape == (12, 21, 40)
    assert np.array_equal(bp[:, :, 0], bp[:, :, -2]) and np.array_equal(bp[:, :, -1], bp[:, :, 1])
    sc = field_scales(m)
    assert [len(s) for s in sc["bp"]] == [12, 21, 40]
    assert [len(s) for s in sc["br"]] == [11, 21, 41]


class _OracleSolver:
    """Stands in for the GPU solver so the driver's host flow (namelist,
    files, lines) can run on CPU; every number comes from the oracle."""

    def __init__(self, mesh, br0, option="ss", ifprec=1, precision="fp64", br1=None, device=-1):
        import oracle as O
        self.mesh = mesh
        mo = O.Mesh(mesh.nr, mesh.nt, mesh.np, *[getattr(mesh, f) for f in O.MESH_FIELDS])
        self.o = O.Solver(mo, br0, option, ifprec, br1=br1)
        self.N = self.o.N
        self.last_info = None
        self._hist = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def rhs(self):
        return self.o.rhs()

    def cgsolve(self, x, r, ncgmax=10_000_000, epscg=1e-9):
        from types import SimpleNamespace
        out = self.o.cgsolve(x, r, ncgmax=ncgmax, epscg=epscg, ncghist=1)
        x[:] = out["x"]
        r[:] = out["r"]
        self._hist = [e for _, e in out["history"]]
        self.last_info = SimpleNamespace(ncg=out["ncg"], epsn=out["epsn"], seconds=0.0)
        return out["ierr"]

    def history(self):
        return np.array(self._hist)

    def fields(self, x, want=("phi", "br", "bt", "bp", "w")):
        phi = self.o.finalize_phi(x)
        br, bt, bp = self.o.getb(phi)
        full = {"phi": phi, "br": br, "bt": bt, "bp": bp, "w": self.o.energy(phi)}
        return {k: full[k] for k in want}


def _dat(path, body):
    path.write_text(" &topology\n" + body[0] + "\n /\n &inputvars\n" + body[1] + "\n /\n")


def test_driver_flow_on_cpu(tmp_path, monkeypatch):
    import pot3d_b200.solver as S
    from pot3d_b200.run import run
    monkeypatch.setattr(S, "Pot3dSolver", _OracleSolver)
    tn, pn, fi = host.synthetic_br(4, 6, 2, 19, 37)
    write_psi(tmp_path / "map.h5", fi, [tn, pn])
    _dat(tmp_path / "pot3d.dat", ("  nr=10\n  nt=17\n  np=29",
                                  "  option='open'\n  br0file='map.h5'\n  r1=2.5\n  rfrac=0.0,1.0\n  drratio=2.5\n"
                                  "  do_not_balance_flux=.true.\n  phifile='phi.h5'\n  br_photo_original_file='orig.h5'\n"
                                  "  hdf32=.false.\n  ncghist=10\n  epscg=1.e-10"))
    res = run(str(tmp_path / "pot3d.dat"), quiet=True)
    m = host.mesh_from_namelist(namelist.read(str(tmp_path / "pot3d.dat")))
    br0 = host.br0_from_map(m, tn, pn, fi, option="open", do_not_balance_flux=True)
    assert np.array_equal(read_psi(tmp_path / "br_photo.h5").data, br0)
    orig = read_psi(tmp_path / "orig.h5").data
    assert np.array_equal(np.abs(orig), br0) and np.any(orig < 0)
    phi = read_psi(tmp_path / "phi.h5")
    assert phi.data.shape == (10, 17, 29) and np.array_equal(phi.scales[0], m.rh)
    for f, shape in (("br", (9, 17, 29)), ("bt", (10, 16, 29)), ("bp", (10, 17, 28))):
        assert read_psi(tmp_path / f"{f}.h5").data.shape == shape
    out = (tmp_path / "pot3d.out").read_text().splitlines()
    assert out[-4:] == _energy_lines(res["energy"])
    assert " ### The CG solver has converged." in out
    assert f" Number of iterations = {res['ncg']:12d}" in out


def test_driver_validation_flow_on_cpu(tmp_path, monkeypatch):
    import pot3d_b200.solver as S
    from pot3d_b200.run import run
    monkeypatch.setattr(S, "Pot3dSolver", _OracleSolver)
    errs = []
    for nr, nt, np_ in ((12, 21, 41), (22, 41, 81)):
        d = tmp_path / str(nr)
        d.mkdir()
        _dat(d / "pot3d.dat", (f"  nr={nr}\n  nt={nt}\n  np={np_}",
                               "  option='ss'\n  validation_run=.true.\n  r1=2.5\n  rfrac=0.0,1.0\n  drratio=2.5\n"
                               "  ncghist=0\n  epscg=1.e-11\n  hdf32=.true."))
        res = run(str(d / "pot3d.dat"), quiet=True)
        errs.append(res["validation_rel_l2"])
        assert read_psi(d / "br_solved.h5").dtype == np.float64  # validation forces hdf32 off
        assert read_psi(d / "phi_exact.h5").data.shape == (nr, nt, np_)
    assert errs[1]["br"] < errs[0]["br"] / 3.5 and errs[1]["bt"] < errs[0]["bt"] / 3.5
    assert errs[1]["bp"] < errs[0]["bp"] / 1.8


def test_driver_rejects_more_than_one_process(tmp_path):
    from pot3d_b200.run import run
    _dat(tmp_path / "pot3d.dat", ("  nprocs=2,1,1\n  nr=10\n  nt=17\n  np=29", "  option='ss'"))
    with pytest.raises(namelist.NamelistError):
        run(str(tmp_path / "pot3d.dat"), quiet=True)
