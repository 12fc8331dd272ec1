"""Reader for POT3D's ``pot3d.dat`` input namelists.

The reference reads two Fortran namelist groups, ``&topology`` and
``&inputvars`` (read_input_file, src/pot3d.F90:827-1003), with defaults from
its modules (cgcom src/pot3d.F90:428-431, vars :462-497, meshdef :355-380).
This parser accepts the subset those groups use -- integers, reals, logicals,
quoted strings and comma-separated arrays, ``!`` comments -- and returns the
values with the reference's defaults filled in.  Unknown keys are an error,
as they are for a Fortran namelist read.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

NMSEG = 30  # meshdef, src/pot3d.F90:365


def _defaults():
    return {
        # &topology
        "nprocs": [-1, -1, -1], "nr": None, "nt": None, "np": None,
        # &inputvars (vars, meshdef, cgcom, global_mesh, debug modules)
        "outfile": "pot3d.out", "phifile": "default", "br0file": "default", "brfile": "default",
        "btfile": "default", "bpfile": "default", "br_photo_file": "default",
        "br_photo_original_file": "default", "option": "potential", "ndump": 0,
        "do_not_balance_flux": False, "fmt": "h5", "hdf32": True, "validation_run": False,
        "dipole_angle": 0.7853981633974483, "r0": 1.0, "r1": 30.0,
        "drratio": [0.0] * NMSEG, "dtratio": [0.0] * NMSEG, "dpratio": [0.0] * NMSEG,
        "rfrac": [0.0] * NMSEG, "tfrac": [0.0] * NMSEG, "pfrac": [0.0] * NMSEG,
        "nfrmesh": 0, "nftmesh": 0, "nfpmesh": 0, "phishift": 0.0,
        "ifprec": 1, "ncgmax": 1000000, "ncghist": 100, "epscg": 1.e-9, "idebug": 0,
    }


_ARRAYS = {"nprocs", "drratio", "dtratio", "dpratio", "rfrac", "tfrac", "pfrac"}
_INTS = {"nr", "nt", "np", "ndump", "nfrmesh", "nftmesh", "nfpmesh", "ifprec", "ncgmax", "ncghist", "idebug"}
_BOOLS = {"do_not_balance_flux", "hdf32", "validation_run"}
_STRS = {"outfile", "phifile", "br0file", "brfile", "btfile", "bpfile", "br_photo_file",
         "br_photo_original_file", "option", "fmt"}


class NamelistError(ValueError):
    pass


def _scalar(tok: str):
    t = tok.strip()
    if not t:
        return None
    if t[0] in "'\"":
        return t[1:-1]
    tl = t.lower()
    if tl in (".true.", ".t.", "t"):
        return True
    if tl in (".false.", ".f.", "f"):
        return False
    t2 = re.sub(r"(?i)(?<=[0-9.])d", "e", t)
    t2 = re.sub(r"(?i)_r_typ$", "", t2)
    try:
        return int(t2)
    except ValueError:
        return float(t2)


def _split_values(s: str):
    out, cur, q = [], "", None
    for ch in s:
        if q:
            cur += ch
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            cur += ch
        elif ch == ",":
            out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur)
    return [v for v in (x.strip() for x in out) if v != ""]


@dataclass
class Pot3dInput:
    values: dict = field(default_factory=_defaults)

    def __getattr__(self, k):
        try:
            return self.__dict__["values"][k]
        except KeyError as e:
            raise AttributeError(k) from e

    @property
    def pm_r1(self) -> float:
        """Boundary switch at r=R1 (check_input, src/pot3d.F90:1250-1285)."""
        opt = self.values["option"].strip()
        if opt == "potential":
            return 1.0
        if opt in ("open", "ss"):
            return -1.0
        raise NamelistError(f"Invalid OPTION: {opt}")


def parse(text: str) -> Pot3dInput:
    """Parse pot3d.dat text into a Pot3dInput with reference defaults."""
    lines = []
    for ln in text.splitlines():
        q, buf = None, ""
        for ch in ln:
            if q:
                buf += ch
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
                buf += ch
            elif ch == "!":
                break
            else:
                buf += ch
        lines.append(buf)
    body = "\n".join(lines)
    vals = _defaults()
    groups = re.findall(r"&(\w+)(.*?)/", body, flags=re.S)
    if not groups:
        raise NamelistError("no namelist groups found")
    for gname, content in groups:
        if gname.lower() not in ("topology", "inputvars"):
            raise NamelistError(f"unknown namelist group &{gname}")
        # split into key=value assignments
        parts = re.split(r"(?:^|\s|,)(\w+(?:\(\d+\))?)\s*=", " " + content)
        for key, val in zip(parts[1::2], parts[2::2]):
            m = re.match(r"(\w+)(?:\((\d+)\))?", key)
            k = m.group(1).lower()
            idx = int(m.group(2)) if m.group(2) else None
            if k not in vals:
                raise NamelistError(f"unknown namelist variable {k}")
            items = [_scalar(v) for v in _split_values(val.replace("\n", " "))]
            if k in _ARRAYS:
                arr = list(vals[k])
                start = (idx - 1) if idx else 0
                for n, v in enumerate(items):
                    arr[start + n] = float(v) if k != "nprocs" else int(v)
                vals[k] = arr
            else:
                if len(items) != 1:
                    raise NamelistError(f"{k} expects one value")
                v = items[0]
                if k in _INTS:
                    v = int(v)
                elif k in _BOOLS:
                    v = bool(v)
                elif k in _STRS:
                    v = str(v)
                else:
                    v = float(v)
                vals[k] = v
    for k in ("nr", "nt", "np"):
        if vals[k] is None:
            raise NamelistError(f"&topology is missing {k}")
    return Pot3dInput(vals)


def read(path) -> Pot3dInput:
    with open(path) as fh:
        return parse(fh.read())
