"""pot3d_gpu_energy_noalloc: the energy diagnostic for callers that cannot
allocate device memory (their memory belongs to another allocator or pool,
or their device footprint is fixed at start-up).  It must give the same
energies as pot3d_gpu_energy, call after call, while the library allocates
nothing for it.  This file is collected last so a stop at the first failure
has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from pot3d_b200 import _lib, host
from pot3d_b200.solver import Pot3dSolver

pytestmark = pytest.mark.gpu


def _fn():
    L = _lib.lib()
    f = L.pot3d_gpu_energy_noalloc
    f.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 10 + [C.c_void_p]
    f.restype = C.c_int
    return f


def test_energy_noalloc_matches_energy_on_two_calls(cuda):
    import torch

    mesh = host.make_mesh(37, 30, 26)
    tn, pn, fi = host.synthetic_br(4, 15, 4, 30, 26)
    br0 = host.br0_from_map(mesh, tn, pn, fi)
    rng = np.random.default_rng(11)
    with Pot3dSolver(mesh, br0) as s:
        phis = [s.finalize_phi(rng.standard_normal(s.N)) for _ in range(2)]
        refs = [s.energy(p) for p in phis]
    dev = {k: torch.tensor(getattr(mesh, k), device=cuda) for k in ("rh", "dr", "drh", "dt", "dth", "sth", "dp", "dph")}
    f = _fn()
    names = ("rh", "dr", "drh", "dt", "dth", "sth", "dp", "dph")
    phs = [torch.tensor(np.asfortranarray(p).ravel(order="F"), device=cuda) for p in phis]
    ws = [torch.full((3,), float("nan"), dtype=torch.float64, device=cuda) for _ in phis]
    torch.cuda.synchronize()
    free = []
    for ph, w, ref in zip(phs, ws, refs):
        rc = f(mesh.nr, mesh.nt, mesh.np, *[C.c_void_p(dev[k].data_ptr()) for k in names],
               C.c_void_p(ph.data_ptr()), C.c_void_p(w.data_ptr()), None)
        assert rc == 0, _lib.lib().pot3d_gpu_last_error()
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        got = w.cpu().numpy()
        assert np.all(np.abs(got - ref) <= 1e-12 * np.abs(ref)), (got, ref)
    # Ten more calls leave the device's free memory unchanged.  The first call
    # may load the library's device code (which holds the scratch array) under
    # lazy module loading, so the count starts after it; mem_get_info counts
    # in pages, so this shows no allocation of a page or more.
    for _ in range(10):
        rc = f(mesh.nr, mesh.nt, mesh.np, *[C.c_void_p(dev[k].data_ptr()) for k in names],
               C.c_void_p(phs[0].data_ptr()), C.c_void_p(ws[0].data_ptr()), None)
        assert rc == 0, _lib.lib().pot3d_gpu_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] >= free[0]
    assert free[1] >= free[0]
    got = ws[0].cpu().numpy()
    assert np.all(np.abs(got - refs[0]) <= 1e-12 * np.abs(refs[0]))


def test_energy_noalloc_rejects_oversized_mesh(cuda):
    f = _fn()
    one = C.c_void_p(1)
    rc = f(10, 10, 8192 + 3, *([one] * 10), None)
    assert rc == 1
    assert b"exceeds the scratch limit" in _lib.lib().pot3d_gpu_last_error()


def test_energy_noalloc_in_a_captured_graph(cuda):
    """After a first call on the device, a call captured into a CUDA graph on
    a non-default stream replays on a new phi written into the captured
    buffer and gives pot3d_gpu_energy's energies of that phi."""
    import torch

    mesh = host.make_mesh(37, 30, 26)
    tn, pn, fi = host.synthetic_br(4, 15, 4, 30, 26)
    br0 = host.br0_from_map(mesh, tn, pn, fi)
    rng = np.random.default_rng(12)
    with Pot3dSolver(mesh, br0) as s:
        phis = [s.finalize_phi(rng.standard_normal(s.N)) for _ in range(3)]
        refs = [s.energy(p) for p in phis]
    names = ("rh", "dr", "drh", "dt", "dth", "sth", "dp", "dph")
    dev = {k: torch.tensor(getattr(mesh, k), device=cuda) for k in names}
    ptrs = [C.c_void_p(dev[k].data_ptr()) for k in names]
    f = _fn()
    ph = torch.tensor(np.asfortranarray(phis[0]).ravel(order="F"), device=cuda)
    w = torch.full((3,), float("nan"), dtype=torch.float64, device=cuda)
    rc = f(mesh.nr, mesh.nt, mesh.np, *ptrs, C.c_void_p(ph.data_ptr()), C.c_void_p(w.data_ptr()), None)
    assert rc == 0, _lib.lib().pot3d_gpu_last_error()
    torch.cuda.synchronize()
    assert np.all(np.abs(w.cpu().numpy() - refs[0]) <= 1e-12 * np.abs(refs[0]))
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(device=cuda)
    with torch.cuda.graph(g, stream=side):
        stream = torch.cuda.current_stream().cuda_stream
        assert stream != 0
        rc = f(mesh.nr, mesh.nt, mesh.np, *ptrs, C.c_void_p(ph.data_ptr()), C.c_void_p(w.data_ptr()),
               C.c_void_p(stream))
    assert rc == 0, _lib.lib().pot3d_gpu_last_error()
    for p, ref in zip(phis[1:], refs[1:]):
        ph.copy_(torch.tensor(np.asfortranarray(p).ravel(order="F"), device=cuda))
        w.fill_(float("nan"))
        g.replay()
        torch.cuda.synchronize()
        got = w.cpu().numpy()
        assert np.all(np.abs(got - ref) <= 1e-12 * np.abs(ref)), (got, ref)
    del g
