"""ctypes binding of libpot3d_gpu.so (include/pot3d_gpu.h, include/pot3d_host.h).

The library is built in-tree by pot3d_b200.build.  There is no fallback: if
the shared library is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpot3d_gpu.so")

_lib = None

MESH_FIELDS = ("r", "dr", "rh", "drh", "t", "dt", "st", "th", "dth", "sth", "p", "dp", "ph", "dph")

GPU_SYMBOLS = (
    "load_external_lu_solver", "external_lu_solver", "unload_external_lu_solver",
    "pot3d_gpu_create", "pot3d_gpu_destroy", "pot3d_gpu_size", "pot3d_gpu_rhs", "pot3d_gpu_cgsolve",
    "pot3d_gpu_cgsolve_dev", "pot3d_gpu_history", "pot3d_gpu_finalize_phi", "pot3d_gpu_energy", "pot3d_gpu_fields",
    "pot3d_gpu_ax_dev", "pot3d_gpu_prec_dev", "pot3d_gpu_precond_diag", "pot3d_gpu_last_error",
    "pot3d_gpu_time_kernels", "pot3d_gpu_time_sweeps", "pot3d_gpu_set_refine", "pot3d_gpu_refine_info", "pot3d_gpu_test_sweep_stall", "pot3d_gpu_set_br0", "pot3d_gpu_br0_from_map", "pot3d_gpu_batch_create", "pot3d_gpu_batch_create_ex", "pot3d_gpu_batch_create_mode", "pot3d_gpu_batch_set_guess", "pot3d_gpu_batch_tune2", "pot3d_gpu_batch_tune", "pot3d_gpu_batch_solve",
    "pot3d_gpu_batch_solution", "pot3d_gpu_batch_destroy",
)
HOST_SYMBOLS = ("pot3d_host_genmesh", "pot3d_host_mesh", "pot3d_host_br0", "pot3d_host_synthetic_br")


class MeshC(C.Structure):
    """pot3d_mesh_t / pot3d_mesh_buf_t (identical layouts)."""
    _fields_ = [("nr", C.c_int), ("nt", C.c_int), ("np", C.c_int)] + [(f, C.c_void_p) for f in MESH_FIELDS]


class SolveInfo(C.Structure):
    """pot3d_solve_info_t."""
    _fields_ = [("ncg", C.c_int), ("n_refine", C.c_int), ("epsn", C.c_double), ("true_resid", C.c_double),
                ("seconds", C.c_double), ("kernel_launches", C.c_longlong)]


class Pot3dError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pot3d_gpu error {code}: {msg}")
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m pot3d_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, dp, fp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int)
        if hasattr(L, "load_external_lu_solver"):
            L.load_external_lu_solver.argtypes = [vp, vp, vp, C.c_int, C.c_int]
            L.load_external_lu_solver.restype = None
            L.external_lu_solver.argtypes = [vp]
            L.external_lu_solver.restype = None
            L.unload_external_lu_solver.argtypes = []
            L.unload_external_lu_solver.restype = None
        L.pot3d_gpu_create.argtypes = [C.POINTER(MeshC), dp, dp, C.c_double, C.c_int, C.c_int, C.c_int,
                                       C.POINTER(vp)]
        L.pot3d_gpu_destroy.argtypes = [vp]
        L.pot3d_gpu_size.argtypes = [vp]
        L.pot3d_gpu_size.restype = C.c_long
        L.pot3d_gpu_rhs.argtypes = [vp, dp]
        L.pot3d_gpu_cgsolve.argtypes = [vp, dp, dp, C.c_long, C.c_int, C.c_double, ip, C.POINTER(SolveInfo)]
        L.pot3d_gpu_cgsolve_dev.argtypes = [vp, vp, vp, C.c_long, C.c_int, C.c_double, ip, C.POINTER(SolveInfo)]
        L.pot3d_gpu_history.argtypes = [vp, dp, C.c_int]
        L.pot3d_gpu_finalize_phi.argtypes = [vp, dp, dp]
        L.pot3d_gpu_energy.argtypes = [vp, dp, dp]
        L.pot3d_gpu_fields.argtypes = [vp, dp, dp, dp, dp, dp, dp]
        L.pot3d_gpu_ax_dev.argtypes = [vp, vp, vp]
        L.pot3d_gpu_prec_dev.argtypes = [vp, vp]
        L.pot3d_gpu_precond_diag.argtypes = [vp, fp, fp]
        L.pot3d_gpu_last_error.restype = C.c_char_p
        L.pot3d_gpu_time_kernels.argtypes = [vp, C.c_int, dp, dp]
        L.pot3d_gpu_time_sweeps.argtypes = [vp, C.c_int, dp]
        L.pot3d_gpu_set_refine.argtypes = [vp, C.c_double, C.c_double, C.c_int]
        L.pot3d_gpu_refine_info.argtypes = [vp, ip, ip]
        L.pot3d_gpu_test_sweep_stall.argtypes = [vp, C.c_uint]
        L.pot3d_gpu_set_br0.argtypes = [vp, dp]
        L.pot3d_gpu_br0_from_map.argtypes = [vp, C.c_int, C.c_int, dp, dp, dp, C.c_int, C.c_int, dp]
        L.pot3d_gpu_batch_create.argtypes = [C.c_int, C.POINTER(MeshC), C.POINTER(dp), dp, C.c_int, C.POINTER(vp)]
        L.pot3d_gpu_batch_create_ex.argtypes = [C.c_int, C.POINTER(MeshC), C.POINTER(dp), dp, C.c_int, C.c_int,
                                                C.POINTER(vp)]
        L.pot3d_gpu_batch_create_mode.argtypes = [C.c_int, C.POINTER(MeshC), C.POINTER(dp), dp, C.c_int, C.c_int,
                                                  C.c_int, C.POINTER(vp)]
        L.pot3d_gpu_batch_set_guess.argtypes = [vp, C.c_int, dp]
        L.pot3d_gpu_batch_tune2.argtypes = [vp, ip, C.c_int, ip, C.c_int, C.c_int, ip, ip, fp]
        L.pot3d_gpu_batch_tune.argtypes = [vp, ip, C.c_int, C.c_int, ip, fp]
        L.pot3d_gpu_batch_solve.argtypes = [vp, C.c_int, C.c_double, ip, C.POINTER(SolveInfo), dp]
        L.pot3d_gpu_batch_solution.argtypes = [vp, C.c_int, dp]
        L.pot3d_gpu_batch_destroy.argtypes = [vp]
        L.pot3d_host_genmesh.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, dp, dp, C.c_int, C.c_int,
                                         C.c_double, dp]
        L.pot3d_host_mesh.argtypes = [C.POINTER(MeshC), C.c_double, C.c_double, C.c_int, dp, dp, C.c_int, dp, dp,
                                      C.c_int, dp, dp, C.c_int, C.c_double]
        L.pot3d_host_br0.argtypes = [C.POINTER(MeshC), C.c_int, C.c_int, dp, dp, dp, C.c_int, C.c_int, dp]
        L.pot3d_host_synthetic_br.argtypes = [C.c_ulonglong, C.c_int, C.c_int, C.c_int, C.c_int, dp, dp, dp]
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != 0:
        raise Pot3dError(code, lib().pot3d_gpu_last_error().decode())


def dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))
