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


# Shapes of the learned operator's GEMMs at 255x361x721 (359 x 719 theta-phi
# positions) and a square reference shape.
BENCH_SHAPES = ((258121, 32, 64, "lift and pointwise layers"), (258121, 128, 64, "first projection"),
                (258121, 128, 128, "radial projection (128 channels)"), (8192, 8192, 8192, "square"))


def main(argv=None):
    """Throughput of tc_gemm (CUDA events, 3 warm-up and 20 timed launches)
    at the operator's shapes, beside torch.matmul on the same operands; with
    --one, a single 8192^3 product after warm-up (for a profiler)."""
    import argparse
    import json

    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--one", action="store_true")
    args = ap.parse_args(argv)
    if args.one:
        A = torch.randn(8192, 8192, device="cuda").bfloat16()
        B = torch.randn(8192, 8192, device="cuda").bfloat16()
        out = torch.empty(8192, 8192, device="cuda", dtype=torch.float32)
        for _ in range(3):
            tc_gemm(A, B, out=out)
        torch.cuda.synchronize()
        check_errors()
        return 0

    def timed(fn, reps=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    for M, N, K, name in BENCH_SHAPES:
        A = torch.randn(M, K, device="cuda").bfloat16()
        B = torch.randn(N, K, device="cuda").bfloat16()
        out = torch.empty(M, N, device="cuda", dtype=torch.float32)
        ms = timed(lambda: tc_gemm(A, B, out=out))
        ref = timed(lambda: torch.matmul(A, B.T))
        check_errors()
        flops, nbytes = 2.0 * M * N * K, 2.0 * (M * K + N * K) + 4.0 * M * N
        print(json.dumps(dict(shape=[M, N, K], name=name, ms=ms, tflops=flops / ms / 1e9, gbs=nbytes / ms / 1e6,
                              torch_ms=ref, torch_tflops=flops / ref / 1e9)), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
