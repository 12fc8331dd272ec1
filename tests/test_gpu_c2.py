"""Parity on the full 255x361x721 PFSS workload (seed 2, 65.3 M unknowns)
against the oracle's own solve of it (tests/golden/pfss_255x361x721_oracle_
ifprec2.*: the reference's CPU PCG with ILU(0) to 1e-11, made once by
tests/golden/make_c2_oracle.py).  Both GPU arithmetic modes, solved to
1e-11: energies within 1e-9 relative, phi on the fixture's three radial
surfaces within 1e-8 relative L2, iteration counts next to the oracle's."""
import json
import os

import numpy as np
import pytest

from conftest import GOLD
from pot3d_b200 import host
from pot3d_b200.solver import Pot3dSolver

pytestmark = pytest.mark.gpu


def _fixture():
    stem = os.path.join(GOLD, "pfss_255x361x721_oracle_ifprec2")
    with open(stem + ".json") as fh:
        rec = json.load(fh)
    z = np.load(stem + ".npz")
    return rec, z["phi_slices"], [int(i) for i in z["slice_i"]], int(z["stride"])


@pytest.mark.parametrize("precision", ["fp32_refined", "fp64"])
def test_full_workload_matches_the_oracle(cuda, precision):
    import torch
    rec, slices, slice_i, stride = _fixture()
    w = host.WORKLOADS["pfss_255x361x721"]
    mesh, br0 = host.pfss_case(w["nr"], w["nt"], w["np"], w["lmax"], w["nbip"], w["seed"])
    with Pot3dSolver(mesh, br0, ifprec=2, precision=precision) as s:
        b = torch.tensor(s.rhs(), device=cuda)
        x = torch.zeros_like(b)
        r = b.clone()
        assert s.cgsolve_dev(x, r, epscg=1e-11, ncgmax=20000) == 0
        ncg = s.last_info.ncg
        out = s.fields(x.cpu().numpy(), want=("phi", "w"))
    wo = np.asarray(rec["energy"])
    assert np.all(np.abs(out["w"] - wo) <= 1e-9 * np.abs(wo)), (out["w"], wo)
    sl = np.stack([out["phi"][i - 1, ::stride, ::stride] for i in slice_i])
    assert np.linalg.norm(sl - slices) <= 1e-8 * np.linalg.norm(slices)
    if precision == "fp64":
        assert abs(ncg - rec["iterations"]) <= 2, (ncg, rec["iterations"])
    else:
        assert ncg <= 1.05 * rec["iterations"], (ncg, rec["iterations"])
