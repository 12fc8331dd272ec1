"""POT3D's program flow for one solve, on the GPU solver.

    python -m pot3d_b200.run [pot3d.dat] [--dir RUN_DIR] [--ifprec 1|2]
                             [--precision fp64|fp32_refined] [--quiet]

Follows the reference's main program (src/pot3d.F90:700-826) for a run on
one GPU: read the namelist (read_input_file :827-1003), build the mesh
(set_global_mesh :2583-2708), read and interpolate the Br map and balance
its flux (readbr + set_flux :3754-3864) or, for a validation run, set the
tilted-dipole boundary fields (set_validation_flux :3978-4066) and write
the analytic solution (write_validation_solution :4068-4131), solve
(potfld :3866-3976), compute B (getb :6187-6233), write the requested
fields as PSI HDF5 files (write_solution :6015-6185) and print the magnetic
energies (magnetic_energy :6235-6321).  The convergence history, the
iteration count and the energies are printed and written to ``outfile`` in
the reference's format.  File names in the namelist are relative to the run
directory (the directory of pot3d.dat unless --dir is given), as the
reference's are relative to its working directory.

Differences from the reference program: one process (nprocs must be unset
or 1 in each direction), no timing.out, and ``--ifprec`` / ``--precision``
may override the namelist's preconditioner and select the FP32-refined
inner solver.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

from . import host, namelist
from .psi_io import read_psi, write_psi

_FIELDS = ("phi", "br", "bt", "bp")


def output_names(v: dict) -> dict:
    """Output file names after the reference's defaults (read_input_file,
    src/pot3d.F90:966-988: 'default' becomes '<name>.<fmt>') and the
    validation-run overrides (:759-790).  An empty name is not written."""
    fmt = v["fmt"].strip()
    names = {}
    for key, base in (("phifile", "phi"), ("brfile", "br"), ("btfile", "bt"), ("bpfile", "bp"),
                      ("br_photo_file", "br_photo"), ("br_photo_original_file", "br_photo_original")):
        nm = v[key].strip()
        names[key] = f"{base}.{fmt}" if nm == "default" else nm
    if v["validation_run"]:
        for key, base in (("phifile", "phi"), ("brfile", "br"), ("btfile", "bt"), ("bpfile", "bp")):
            names[key] = f"{base}_solved.{fmt}"
    names["outfile"] = v["outfile"].strip()
    return names


def field_scales(mesh: host.Mesh) -> dict:
    """The scales write_solution gives each field (src/pot3d.F90:6070-6183)."""
    p = mesh.p[:mesh.np - 1]
    return {"phi": (mesh.rh, mesh.th, mesh.ph), "br": (mesh.r, mesh.th, mesh.ph),
            "bt": (mesh.rh, mesh.t, mesh.ph), "bp": (mesh.rh, mesh.th, p)}


def _energy_lines(w) -> list:
    # magnetic_energy prints with (A,ES22.16), src/pot3d.F90:6273,6306-6309
    return [f"Energy in Br**2 = {w[0]:.16E}", f"Energy in Bt**2 = {w[1]:.16E}",
            f"Energy in Bp**2 = {w[2]:.16E}", f"Magnetic energy = {sum(w):.16E}"]


def _history_lines(hist, ncghist: int, epscg: float) -> list:
    """The lines ernorm writes to outfile (src/pot3d.F90:4433-4458): a line
    every ncghist iterations, then the converged message and the last
    iteration again."""
    out = []
    n = len(hist)
    if ncghist <= 0 or n == 0:
        return out

    def line(it):
        return f" Iteration: {it:8d}   Residual: {hist[it]:23.15E}"

    for it in range(n):
        if it % ncghist == 0:
            if it == 0:
                out += [" ", " ### Convergence information:"]
            out.append(line(it))
    if hist[n - 1] < epscg:
        out += [" ", " ### The CG solver has converged.", line(n - 1)]
    return out


def run(dat_path: str, run_dir: str | None = None, ifprec: int | None = None, precision: str = "fp64",
        quiet: bool = False) -> dict:
    """One POT3D run; returns the energies, iterations, the solver info and
    the written file paths."""
    from .solver import Pot3dSolver
    nml = namelist.read(dat_path)
    v = nml.values
    run_dir = os.path.dirname(os.path.abspath(dat_path)) if run_dir is None else run_dir
    for n in v["nprocs"]:
        if n not in (-1, 1):
            raise namelist.NamelistError("this driver runs one process: nprocs must be unset or 1")
    names = output_names(v)
    lines = []

    def say(*ls):
        lines.extend(ls)
        if not quiet:
            for ln in ls:
                print(ln)

    def path(nm):
        return nm if os.path.isabs(nm) else os.path.join(run_dir, nm)

    labels = {"phifile": "the potential", "brfile": "Br", "btfile": "Bt", "bpfile": "Bp",
              "br_photo_file": "BR0", "br_photo_original_file": "BR0 (before sign flip)"}

    def write(key, data, scales, hdf32):
        if names.get(key, ""):
            write_psi(path(names[key]), data, scales, hdf32=hdf32)
            say(" ", f" Writing {labels[key]} to file: {names[key]}")
            written[key] = path(names[key])

    written = {}
    mesh = host.mesh_from_namelist(nml)
    hdf32 = bool(v["hdf32"])
    option = v["option"].strip()
    nml.pm_r1  # raises NamelistError on an invalid option
    br1 = None
    if v["validation_run"]:
        hdf32 = False
        br0, br1 = host.validation_br(mesh, v["dipole_angle"], v["r0"], v["r1"])
        say(" ", " ### COMMENT from POT3D:", " ### Validation run requested.")
    else:
        d = read_psi(path(v["br0file"].strip()))
        if d.data.ndim != 2 or not d.has_scales:
            raise ValueError(f"{v['br0file']}: a 2-D Br map with theta and phi scales is required")
        if option == "open" and names["br_photo_original_file"]:
            orig = host.br0_from_map(mesh, d.scales[0], d.scales[1], d.data, option="ss",
                                     do_not_balance_flux=v["do_not_balance_flux"])
            write("br_photo_original_file", orig, (mesh.th, mesh.ph), hdf32)
        br0 = host.br0_from_map(mesh, d.scales[0], d.scales[1], d.data, option=option,
                                do_not_balance_flux=v["do_not_balance_flux"])
        write("br_photo_file", br0, (mesh.th, mesh.ph), hdf32)
    ifp = v["ifprec"] if ifprec is None else ifprec
    with Pot3dSolver(mesh, br0, option=option, ifprec=ifp, precision=precision, br1=br1) as s:
        if v["validation_run"]:
            x_ex, br_ex, bt_ex, bp_ex = host.validation_exact(mesh, v["dipole_angle"])
            phi_ex = s.fields(x_ex, want=("phi",))["phi"]
            sc = field_scales(mesh)
            for key, arr in (("phi", phi_ex), ("br", br_ex), ("bt", bt_ex), ("bp", bp_ex)):
                fn = f"{key}_exact.{v['fmt'].strip()}"
                write_psi(path(fn), arr, sc[key], hdf32=False)
                written[f"{key}_exact"] = path(fn)
        say(" ", " ### COMMENT from POT3D:", " ### Starting PCG solve.")
        x = np.zeros(s.N)
        r = s.rhs()
        ierr = s.cgsolve(x, r, ncgmax=v["ncgmax"], epscg=v["epscg"])
        info = s.last_info
        say(*_history_lines(s.history(), v["ncghist"], v["epscg"]))
        if ierr != 0:
            say(" ", " ### ERROR in SOLVE:", " ### The field solver did not converge.",
                f" Number of iterations = {info.ncg:12d}")
            raise RuntimeError(f"PCG did not converge in {info.ncg} iterations (ierr={ierr})")
        say(" ", " ### COMMENT from SOLVE:", " ### The field solver converged.",
            f" Number of iterations = {info.ncg:12d}")
        want = tuple(f for f in _FIELDS if names[f + "file"]) + ("w",)
        if v["validation_run"]:
            want = _FIELDS + ("w",)
        out = s.fields(x, want=want)
        sc = field_scales(mesh)
        for f in _FIELDS:
            if f in out:
                write(f + "file", out[f], sc[f], hdf32)
        w = out["w"]
        say(" ", " ### COMMENT from GETB:", " ### Magnetic energy diagnostic:", " ", *_energy_lines(w))
        res = {"energy": w, "ncg": info.ncg, "epsn": info.epsn, "seconds": info.seconds, "ierr": ierr,
               "files": written, "info": info}
        if v["validation_run"]:
            err = {}
            for f, ex in (("br", br_ex), ("bt", bt_ex), ("bp", bp_ex)):
                sl = (slice(1, -1),) * 3
                err[f] = float(np.linalg.norm((out[f] - ex)[sl]) / np.linalg.norm(ex[sl]))
            res["validation_rel_l2"] = err
            say(" ", " ### Validation: relative L2 error of B against the analytic dipole (interior):",
                *[f" {f}: {e:.6E}" for f, e in err.items()])
    if names["outfile"]:
        with open(path(names["outfile"]), "w") as fh:
            fh.write("\n".join(lines) + "\n")
        res["files"]["outfile"] = path(names["outfile"])
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("dat", nargs="?", default="pot3d.dat")
    ap.add_argument("--dir", default=None, help="run directory for relative file names")
    ap.add_argument("--ifprec", type=int, default=None, choices=(1, 2))
    ap.add_argument("--precision", default="fp64", choices=("fp64", "fp32_refined"))
    ap.add_argument("--quiet", action="store_true")
    a = ap.parse_args(argv)
    try:
        run(a.dat, a.dir, a.ifprec, a.precision, a.quiet)
    except (RuntimeError, ValueError) as e:
        print(f"### ERROR: {e}", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
