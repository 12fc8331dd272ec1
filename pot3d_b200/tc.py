"""Tensor-core GEMM of the learned warm start (pot3d_tc_gemm, tcgen05 BF16).

tc_gemm(A, B) returns A @ B^T for BF16 CUDA tensors shaped [batch, M, K] and
[batch, N, K] (or without the batch axis), accumulating in FP32 on the
tensor cores.  K must be a multiple of 64 and N a multiple of 16.
"""
from __future__ import annotations

import ctypes as C

from . import _lib

_err = {}
# Kernels of the learned path launched so far (GEMMs here, the element-wise
# kernels of fno.py and warmstart.py count themselves).
LAUNCHES = [0]


def _fn():
    L = _lib.lib()
    f = L.pot3d_tc_gemm
    if not getattr(f, "_typed", False):
        f.argtypes = [C.c_void_p] * 4 + [C.c_int] * 4 + [C.c_longlong, C.c_longlong, C.c_int, C.c_int, C.c_void_p,
                                                          C.c_void_p]
        f.restype = C.c_int
        f._typed = True
    return f


def _err_flag(device):
    import torch
    key = str(device)
    if key not in _err:
        _err[key] = torch.zeros(1, dtype=torch.int32, device=device)
    return _err[key]


def tc_gemm(A, B, bias=None, out=None, out_dtype=None, ldd=None, accumulate=False, n=None):
    """out[b, m, :n] (+)= A[b] @ B[b]^T (+ bias).  `out` may be wider than N
    (row stride ldd, e.g. a zero-padded channel buffer)."""
    import torch
    squeeze = A.dim() == 2
    if squeeze:
        A, B = A.unsqueeze(0), B.unsqueeze(0)
        if out is not None:
            out = out.unsqueeze(0)
    assert A.dtype == torch.bfloat16 and B.dtype == torch.bfloat16 and A.is_cuda and B.is_cuda
    assert A.is_contiguous() and B.is_contiguous()
    bsz, M, K = A.shape
    bb, N, K2 = B.shape
    assert bb == bsz and K2 == K
    out_dtype = out_dtype or torch.float32
    if out is None:
        out = torch.zeros((bsz, M, N), dtype=out_dtype, device=A.device) if accumulate else \
            torch.empty((bsz, M, N), dtype=out_dtype, device=A.device)
    assert out.is_contiguous() and out.shape[0] == bsz and out.shape[1] == M
    ldd = out.shape[-1] if ldd is None else ldd
    assert ldd >= N and out.shape[-1] == ldd
    err = _err_flag(A.device)
    stream = torch.cuda.current_stream(A.device).cuda_stream
    rc = _fn()(C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()), C.c_void_p(out.data_ptr()),
               C.c_void_p(bias.data_ptr()) if bias is not None else None, bsz, M, N, K, ldd, M * ldd,
               1 if accumulate else 0, 1 if out.dtype == torch.bfloat16 else 0, C.c_void_p(err.data_ptr()),
               C.c_void_p(stream))
    _lib.check(rc)
    LAUNCHES[0] += 1
    return out[0] if squeeze else out


def check_errors(device="cuda"):
    """Raise if a tensor-core GEMM reported a timed-out wait."""
    e = _err_flag(device)
    if int(e.item()) != 0:
        raise RuntimeError("pot3d_tc_gemm: a bounded wait ran out on the device")
