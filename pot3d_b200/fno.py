"""Learned warm start: a Fourier-style neural operator predicting phi from Br.

The operator maps the boundary map Br0(theta, phi) of one case to its
potential phi(r, theta, phi) on the interior mesh; the radial levels are the
output channels ("r as channel-conditioned depth"), so one pass yields the
whole field in the solver's packed layout (r fastest, then theta, then phi).

Architecture (width 32, 4 Fourier layers, GELU):
    lift 4 -> 32  ->  4 x [ v <- act( W v + b + K(v) ) ]  ->  32 -> 128 -> R
with K the spectral convolution on (theta, phi) slices keeping 16 theta
modes (cosine basis: the even extension of theta over the poles) and 32 phi
coefficients (cos m phi, m = 0..15, and sin m phi, m = 1..16), mixed per
mode by a 32x32 channel matrix.  The truncated transforms are dense products
with precomputed basis matrices, so the whole network is a chain of GEMMs:
every contraction, forward and backward, runs on the tcgen05 tensor-core
GEMM (BF16 operands, FP32 accumulation); layout changes, activations, the
loss and Adam are small kernels of the same library.  Weights are FP32
master copies with BF16 working copies.

Inputs per grid point: Br0/sigma, cos(theta), sin(theta), 1, with sigma the
RMS of Br0; the target is phi/sigma (the solve is linear in Br0), so the
predicted initial guess is sigma times the network output.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from .tc import tc_gemm

F32, BF16 = 0, 1


def _count():
    from .tc import LAUNCHES
    LAUNCHES[0] += 1


def _ceil(n, m):
    return (n + m - 1) // m * m


def _L():
    L = _lib.lib()
    if not getattr(L, "_fno_typed", False):
        vp, ll = C.c_void_p, C.c_longlong
        L.pot3d_fno_permute.argtypes = [vp, C.c_int, C.POINTER(ll), vp, C.c_int, C.POINTER(ll), C.POINTER(C.c_int),
                                        C.c_int, vp]
        L.pot3d_fno_gelu.argtypes = [vp, ll, C.c_int, C.c_int, vp, C.c_int, C.c_int, vp, C.c_int, C.c_int, C.c_int, vp]
        L.pot3d_fno_colsum.argtypes = [vp, ll, C.c_int, C.c_int, vp, C.c_int, vp, C.c_int, vp]
        L.pot3d_fno_relmse.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int, ll, C.c_int, C.c_float, vp, vp, vp]
        L.pot3d_fno_adam.argtypes = [vp, vp, vp, vp, vp, ll, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, vp]
        L.pot3d_fno_inputs.argtypes = [vp, vp, ll, ll, vp, vp]
        L.pot3d_fno_guess.argtypes = [vp, ll, ll, C.c_int, C.c_int, vp, vp, vp]
        L.pot3d_fno_guess_resampled.argtypes = [vp, ll, ll, C.c_int, C.c_int, vp, vp, C.c_int, vp, vp, vp]
        L._fno_typed = True
    return L


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dt(t):
    import torch
    return BF16 if t.dtype == torch.bfloat16 else F32


def permute(inp, in_dims, out, out_dims, perm, add=False):
    """out[o] = inp[i] with i[perm[a]] = o[a]; zero outside inp (pad/crop)."""
    idd = (C.c_longlong * 4)(*in_dims)
    odd = (C.c_longlong * 4)(*out_dims)
    pp = (C.c_int * 4)(*perm)
    _count()
    _lib.check(_L().pot3d_fno_permute(C.c_void_p(inp.data_ptr()), _dt(inp), idd, C.c_void_p(out.data_ptr()),
                                      _dt(out), odd, pp, 1 if add else 0, _stream()))
    return out


def new(shape, dtype="bf16", zero=False):
    import torch
    dt = torch.bfloat16 if dtype == "bf16" else torch.float32
    return (torch.zeros if zero else torch.empty)(shape, dtype=dt, device="cuda")


def act(pre, C_, ldp, out, ldo, mode, grad=None, ldg=0):
    """mode 'gelu': out = gelu(pre); 'dgelu': out = grad * gelu'(pre);
    'copy': out = pre (identity), always zero-padding columns C_..ldo."""
    M = pre.numel() // ldp
    if mode == "copy":
        permute(pre, (1, 1, M, ldp), out, (1, 1, M, ldo), (0, 1, 2, 3))
        return out
    bwd = 1 if mode == "dgelu" else 0
    _count()
    _lib.check(_L().pot3d_fno_gelu(C.c_void_p(pre.data_ptr()), M, C_, ldp,
                                   C.c_void_p(grad.data_ptr()) if grad is not None else None,
                                   _dt(grad) if grad is not None else 0, ldg, C.c_void_p(out.data_ptr()), _dt(out),
                                   ldo, bwd, _stream()))
    return out


def colsum(x, C_, ld, out, add=False, scratch=None):
    M = x.numel() // ld
    scratch = scratch if scratch is not None else new((64 * C_,), "f32")
    _count()
    _lib.check(_L().pot3d_fno_colsum(C.c_void_p(x.data_ptr()), M, C_, ld, C.c_void_p(out.data_ptr()),
                                     1 if add else 0, C.c_void_p(scratch.data_ptr()), scratch.numel(), _stream()))
    return out


def transpose2(x, rows, cols, rows_out=None, cols_out=None, dtype="bf16"):
    """[rows, cols] -> [cols_out, rows_out] (zero padded)."""
    ro = rows_out or rows
    co = cols_out or cols
    out = new((co, ro), dtype)
    permute(x, (1, 1, rows, cols), out, (1, 1, co, ro), (0, 1, 3, 2))
    return out


@dataclass
class Grid:
    nth: int
    nph: int
    R: int
    th: np.ndarray   # interior theta (nth)
    dth: np.ndarray
    ph: np.ndarray   # interior phi (nph)
    dph: np.ndarray


def grid_from_mesh(mesh) -> Grid:
    return Grid(mesh.nt - 2, mesh.np - 2, mesh.nr - 2, mesh.th[1:-1].copy(), mesh.dth[1:-1].copy(),
                mesh.ph[1:-1].copy(), mesh.dph[1:-1].copy())


def radial_weights(rh_src, rh_dst, r0_dst, r1_dst):
    """Linear interpolation from the interior half-mesh levels of rh_src
    (ghosts included; its boundaries sit midway between ghost and first
    point) onto those of rh_dst (boundaries r0_dst, r1_dst), in the radial
    coordinate normalised to [0, 1] between the boundaries: level i of the
    destination is o[idx[i]] + w[i] (o[idx[i]+1] - o[idx[i]]), with w
    outside [0, 1] extrapolating past the first and last source levels."""
    rh_src = np.asarray(rh_src, np.float64)
    r0_src = 0.5 * (rh_src[0] + rh_src[1])
    r1_src = 0.5 * (rh_src[-2] + rh_src[-1])
    s_src = (rh_src[1:-1] - r0_src) / (r1_src - r0_src)
    s_dst = (np.asarray(rh_dst, np.float64)[1:-1] - r0_dst) / (r1_dst - r0_dst)
    idx = np.clip(np.searchsorted(s_src, s_dst) - 1, 0, len(s_src) - 2).astype(np.int32)
    w = (s_dst - s_src[idx]) / (s_src[idx + 1] - s_src[idx])
    return idx, w


def bases(g: Grid, mt=16, mp=32):
    """Forward (analysis) and inverse (synthesis) matrices, padded for the
    GEMM: Ft [mt, Pth], Fp [mp, Pph], Gt [Pth, 64], Gp [Pph, 64]."""
    Pth, Pph = _ceil(g.nth, 64), _ceil(g.nph, 64)
    Ft = np.zeros((mt, Pth))
    Gt = np.zeros((Pth, 64))
    for m in range(mt):
        Ft[m, :g.nth] = np.cos(m * g.th) * g.dth
        Gt[:g.nth, m] = np.cos(m * g.th) * (1.0 / math.pi if m == 0 else 2.0 / math.pi)
    Fp = np.zeros((mp, Pph))
    Gp = np.zeros((Pph, 64))
    half = mp // 2
    for m in range(half):  # cos m phi, m = 0..half-1
        Fp[m, :g.nph] = np.cos(m * g.ph) * g.dph
        Gp[:g.nph, m] = np.cos(m * g.ph) * (1.0 / (2 * math.pi) if m == 0 else 1.0 / math.pi)
    for q in range(half):  # sin m phi, m = 1..half
        m = q + 1
        Fp[half + q, :g.nph] = np.sin(m * g.ph) * g.dph
        Gp[:g.nph, half + q] = np.sin(m * g.ph) / math.pi
    return Ft, Fp, Gt, Gp


class FNO:
    def __init__(self, grid: Grid, width=32, layers=4, mt=16, mp=32, hidden=128, in_ch=4, seed=0):
        import torch
        self.g = grid
        self.W, self.nl, self.mt, self.mp, self.hidden, self.in_ch = width, layers, mt, mp, hidden, in_ch
        self.Pth, self.Pph = _ceil(grid.nth, 64), _ceil(grid.nph, 64)
        self.Rp = _ceil(grid.R, 64)  # output channels; a GEMM K dimension in backward
        self.nmodes = mt * mp
        Ft, Fp, Gt, Gp = bases(grid, mt, mp)
        bf = lambda a: torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).cuda().contiguous()
        self.Ft, self.Fp, self.Gt, self.Gp = bf(Ft), bf(Fp), bf(Gt), bf(Gp)
        # adjoints for the backward pass, K-padded to 64
        FtT = np.zeros((self.Pth, 64)); FtT[:, :mt] = Ft.T
        FpT = np.zeros((self.Pph, 64)); FpT[:, :mp] = Fp.T
        GtT = np.zeros((64, self.Pth)); GtT[:mt, :] = Gt[:, :mt].T
        GpT = np.zeros((64, self.Pph)); GpT[:mp, :] = Gp[:, :mp].T
        self.FtT, self.FpT, self.GtT, self.GpT = bf(FtT), bf(FpT), bf(GtT), bf(GpT)
        rng = np.random.default_rng(seed)
        W_ = width

        def lin(n_out, n_in, kpad, npad=None):
            a = np.zeros((npad or n_out, kpad), np.float32)
            a[:n_out, :n_in] = rng.standard_normal((n_out, n_in)) / math.sqrt(n_in)
            return a
        p = {}
        p["Plift"] = lin(W_, in_ch, 64)
        p["blift"] = np.zeros(W_, np.float32)
        for l in range(layers):
            p[f"W{l}"] = lin(W_, W_, 64)
            p[f"b{l}"] = np.zeros(W_, np.float32)
            r = np.zeros((self.nmodes, W_, 64), np.float32)
            r[:, :, :W_] = rng.standard_normal((self.nmodes, W_, W_)) / W_
            p[f"R{l}"] = r
        p["Q1"] = lin(hidden, W_, 64)
        p["bq1"] = np.zeros(hidden, np.float32)
        p["Q2"] = lin(grid.R, hidden, hidden, npad=self.Rp)
        p["bq2"] = np.zeros(self.Rp, np.float32)
        self.p = {k: torch.tensor(v).cuda().contiguous() for k, v in p.items()}
        self.pb = {k: v.to(torch.bfloat16).contiguous() for k, v in self.p.items() if v.dim() >= 2}
        self.m1 = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.m2 = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.step_count = 0
        self.scratch = new((64 * max(hidden, self.Rp, 64),), "f32")

    # ---------------------------------------------------------------- input
    def inputs(self, br0_list):
        """Network inputs [B, nph, nth, 64] (BF16) and the scales sigma."""
        import torch
        g = self.g
        B = len(br0_list)
        x = np.zeros((B, g.nph, g.nth, 64), np.float32)
        sig = np.zeros(B)
        ct, stt = np.cos(g.th), np.sin(g.th)
        for b, br0 in enumerate(br0_list):
            inner = np.asarray(br0)[1:-1, 1:-1]  # (nth, nph) of the Fortran (nt, np) array
            s = float(np.sqrt(np.mean(inner ** 2))) or 1.0
            sig[b] = s
            x[b, :, :, 0] = (inner / s).T
            x[b, :, :, 1] = ct[None, :]
            x[b, :, :, 2] = stt[None, :]
            x[b, :, :, 3] = 1.0
        return torch.tensor(x).to(torch.bfloat16).cuda().contiguous(), sig

    # -------------------------------------------------------------- forward
    def forward(self, x, keep=False):
        """x [B, nph, nth, 64] BF16 -> prediction [B, nph, nth, Rp] FP32."""
        g, W_ = self.g, self.W
        B = x.shape[0]
        M = B * g.nph * g.nth
        cache = {"x": x, "B": B, "M": M} if keep else None
        pre = tc_gemm(x.view(M, 64), self.pb["Plift"], bias=self.p["blift"])
        v = act(pre, W_, W_, new((M, 64), "bf16"), 64, "copy")
        if keep:
            cache["pre_lift"] = pre
        for l in range(self.nl):
            last = l == self.nl - 1
            st = self._spectral(v, B, cache, l)
            pre = tc_gemm(v, self.pb[f"W{l}"], bias=self.p[f"b{l}"])  # [M, 32]
            permute(st, (B, W_, g.nph, self.Pth), pre, (B, g.nph, g.nth, W_), (0, 2, 3, 1), add=True)
            if keep:
                cache[f"v{l}"] = v
                cache[f"pre{l}"] = pre
            v = act(pre, W_, W_, new((M, 64), "bf16"), 64, "copy" if last else "gelu")
        hpre = tc_gemm(v, self.pb["Q1"], bias=self.p["bq1"])
        h = act(hpre, self.hidden, self.hidden, new((M, self.hidden), "bf16"), self.hidden, "gelu")
        out = tc_gemm(h, self.pb["Q2"], bias=self.p["bq2"])
        if keep:
            cache.update(vL=v, hpre=hpre, h=h)
            self._cache = cache
        return out.view(B, g.nph, g.nth, self.Rp)

    def _spectral(self, v, B, cache=None, l=0):
        """K(v): [B, nph, nth, 64] -> [B, W, nph, Pth] (BF16)."""
        g, W_, mt, mp = self.g, self.W, self.mt, self.mp
        T1 = permute(v, (B, g.nph, g.nth, 64), new((B, W_, g.nph, self.Pth)), (B, W_, g.nph, self.Pth), (0, 3, 1, 2))
        D1 = tc_gemm(T1.view(-1, self.Pth), self.Ft, out_dtype=_bf())  # [B W nph, mt]
        T2 = permute(D1, (B, W_, g.nph, mt), new((B, W_, mt, self.Pph)), (B, W_, mt, self.Pph), (0, 1, 3, 2))
        D2 = tc_gemm(T2.view(-1, self.Pph), self.Fp, out_dtype=_bf())  # [B W mt, mp]
        T3 = permute(D2, (B, W_, mt, mp), new((mt, mp, B, 64)), (mt, mp, B, 64), (2, 3, 0, 1))
        D3 = tc_gemm(T3.view(self.nmodes, B, 64), self.pb[f"R{l}"], out_dtype=_bf())  # [modes, B, W]
        T4 = permute(D3, (mt, mp, B, W_), new((B, W_, mt, 64)), (B, W_, mt, 64), (2, 3, 0, 1))
        D4 = tc_gemm(T4.view(-1, 64), self.Gp, out_dtype=_bf())  # [B W mt, Pph]
        T5 = permute(D4, (B, W_, mt, self.Pph), new((B, W_, g.nph, 64)), (B, W_, g.nph, 64), (0, 1, 3, 2))
        D5 = tc_gemm(T5.view(-1, 64), self.Gt, out_dtype=_bf())  # [B W nph, Pth]
        if cache is not None:
            cache[f"T3_{l}"] = T3
        return D5

    # ------------------------------------------------------------- backward
    def backward(self, dout):
        """dout [B, nph, nth, Rp] FP32 -> gradients (FP32, same shapes as p)."""
        c = self._cache
        g, W_, mt, mp = self.g, self.W, self.mt, self.mp
        B, M = c["B"], c["M"]
        Mp = _ceil(M, 64)
        grads = {}
        dout = dout.view(M, self.Rp)
        dout_b = act(dout, self.Rp, self.Rp, new((M, self.Rp)), self.Rp, "copy")
        grads["Q2"] = tc_gemm(transpose2(dout, M, self.Rp, rows_out=Mp), transpose2(c["h"], M, self.hidden, rows_out=Mp))
        grads["bq2"] = colsum(dout, self.Rp, self.Rp, new((self.Rp,), "f32"), scratch=self.scratch)
        dh = tc_gemm(dout_b, transpose2(self.pb["Q2"], self.Rp, self.hidden))  # [M, hidden]
        dhp = act(c["hpre"], self.hidden, self.hidden, new((M, self.hidden), "f32"), self.hidden, "dgelu",
                  grad=dh, ldg=self.hidden)
        dhp_b = act(dhp, self.hidden, self.hidden, new((M, self.hidden)), self.hidden, "copy")
        grads["Q1"] = tc_gemm(transpose2(dhp, M, self.hidden, rows_out=Mp), transpose2(c["vL"], M, 64, rows_out=Mp))
        grads["bq1"] = colsum(dhp, self.hidden, self.hidden, new((self.hidden,), "f32"), scratch=self.scratch)
        dv = tc_gemm(dhp_b, transpose2(self.pb["Q1"], self.hidden, 64))  # [M, 64]
        for l in reversed(range(self.nl)):
            last = l == self.nl - 1
            pre = c[f"pre{l}"]
            if last:
                dpre = act(dv, W_, 64, new((M, W_), "f32"), W_, "copy")
            else:
                dpre = act(pre, W_, W_, new((M, W_), "f32"), W_, "dgelu", grad=dv, ldg=64)
            dpre_b = act(dpre, W_, W_, new((M, 64)), 64, "copy")
            v = c[f"v{l}"]
            grads[f"W{l}"] = tc_gemm(transpose2(dpre, M, W_, rows_out=Mp), transpose2(v, M, 64, rows_out=Mp))
            grads[f"b{l}"] = colsum(dpre, W_, W_, new((W_,), "f32"), scratch=self.scratch)
            WT = transpose2(self.pb[f"W{l}"], W_, 64, rows_out=64)  # [64 (c), 64 (c' padded)]
            dv_new = tc_gemm(dpre_b, WT)  # [M, 64]
            # spectral path, adjoint chain
            dD5 = permute(dpre, (B, g.nph, g.nth, W_), new((B, W_, g.nph, self.Pth)), (B, W_, g.nph, self.Pth),
                          (0, 3, 1, 2))
            dT5 = tc_gemm(dD5.view(-1, self.Pth), self.GtT, out_dtype=_bf())  # [B W nph, 64]
            dD4 = permute(dT5, (B, W_, g.nph, 64), new((B, W_, mt, self.Pph)), (B, W_, mt, self.Pph), (0, 1, 3, 2))
            dT4 = tc_gemm(dD4.view(-1, self.Pph), self.GpT, out_dtype=_bf())  # [B W mt, 64]
            dD3 = permute(dT4, (B, W_, mt, 64), new((mt, mp, B, 64)), (mt, mp, B, 64), (2, 3, 0, 1))
            T3 = c[f"T3_{l}"]
            Bp = _ceil(B, 64)
            dD3T = permute(dD3, (1, self.nmodes, B, 64), new((1, self.nmodes, W_, Bp)), (1, self.nmodes, W_, Bp),
                           (0, 1, 3, 2))
            T3T = permute(T3, (1, self.nmodes, B, 64), new((1, self.nmodes, 64, Bp)), (1, self.nmodes, 64, Bp),
                          (0, 1, 3, 2))
            grads[f"R{l}"] = tc_gemm(dD3T.view(self.nmodes, W_, Bp), T3T.view(self.nmodes, 64, Bp))
            RT = permute(self.pb[f"R{l}"], (1, self.nmodes, W_, 64), new((1, self.nmodes, 64, 64)),
                         (1, self.nmodes, 64, 64), (0, 1, 3, 2))
            dT3 = tc_gemm(dD3.view(self.nmodes, B, 64), RT.view(self.nmodes, 64, 64), out_dtype=_bf())
            dD2 = permute(dT3, (mt, mp, B, 64), new((B, W_, mt, 64)), (B, W_, mt, 64), (2, 3, 0, 1))
            dT2 = tc_gemm(dD2.view(-1, 64), self.FpT, out_dtype=_bf())  # [B W mt, Pph]
            dD1 = permute(dT2, (B, W_, mt, self.Pph), new((B, W_, g.nph, 64)), (B, W_, g.nph, 64), (0, 1, 3, 2))
            dT1 = tc_gemm(dD1.view(-1, 64), self.FtT, out_dtype=_bf())  # [B W nph, Pth]
            permute(dT1, (B, W_, g.nph, self.Pth), dv_new, (B, g.nph, g.nth, 64), (0, 2, 3, 1), add=True)
            dv = dv_new
        dlift = act(dv, W_, 64, new((M, W_), "f32"), W_, "copy")
        grads["Plift"] = tc_gemm(transpose2(dlift, M, W_, rows_out=Mp), transpose2(c["x"].view(M, 64), M, 64, rows_out=Mp))
        grads["blift"] = colsum(dlift, W_, W_, new((W_,), "f32"), scratch=self.scratch)
        return grads

    # ------------------------------------------------------------- training
    def loss_and_grad(self, x, target):
        """Relative squared error per sample (mean over the batch) and its
        gradient with respect to the prediction."""
        import torch
        B = x.shape[0]
        out = self.forward(x, keep=True)
        npos = self.g.nph * self.g.nth
        grad = torch.empty_like(out)
        loss = new((B,), "f32")
        _count()
        _lib.check(_L().pot3d_fno_relmse(C.c_void_p(out.data_ptr()), self.Rp, C.c_void_p(target.data_ptr()),
                                         _dt(target), B, npos, self.g.R, 1.0 / B, C.c_void_p(grad.data_ptr()),
                                         C.c_void_p(loss.data_ptr()), _stream()))
        return loss, grad

    def adam_step(self, grads, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        for k, w in self.p.items():
            gk = grads[k].contiguous().view(-1)
            assert gk.numel() == w.numel(), k
            wb = self.pb.get(k)
            _count()
            _lib.check(_L().pot3d_fno_adam(C.c_void_p(w.data_ptr()), C.c_void_p(gk.data_ptr()),
                                           C.c_void_p(self.m1[k].data_ptr()), C.c_void_p(self.m2[k].data_ptr()),
                                           C.c_void_p(wb.data_ptr()) if wb is not None else None, w.numel(), lr, b1,
                                           b2, eps, self.step_count, _stream()))

    # ----------------------------------------------------------- weights
    def save(self, path):
        """Parameters as BF16 bits (matrices, the precision inference uses)
        and FP32 (bias vectors), with the grid they were trained on."""
        import torch
        out = {"grid": np.array([self.g.nth, self.g.nph, self.g.R, self.W, self.nl, self.mt, self.mp, self.hidden,
                                 self.in_ch], np.int64)}
        for k, v in self.p.items():
            if v.dim() >= 2:
                out["bf16_" + k] = v.to(torch.bfloat16).view(torch.int16).cpu().numpy()
            else:
                out["f32_" + k] = v.cpu().numpy()
        np.savez_compressed(path, **out)

    @classmethod
    def load(cls, path, grid: "Grid"):
        """A model saved by save() for the same grid (theta, phi, radial sizes)."""
        z = np.load(path)
        nth, nph, R = (int(v) for v in z["grid"][:3])
        if (nth, nph, R) != (grid.nth, grid.nph, grid.R):
            raise ValueError(f"{path}: trained for {nth}x{nph}x{R}, not {grid.nth}x{grid.nph}x{grid.R}")
        return cls._from_saved(path, z, grid)

    @classmethod
    def load_resampled(cls, path, mesh):
        """A model saved by save() applied on the grid of `mesh`, which may
        differ from the training grid: the theta-phi layers are free of the
        resolution (quadrature-weighted truncated bases, pointwise lifts and
        projections), so the network runs on mesh's theta-phi points as it
        is; its radial levels (the output channels, those of the training
        mesh) are interpolated linearly onto mesh's in the radial coordinate
        normalised to [0, 1] between the inner and outer radius.  The
        training mesh's half-mesh radii are the file's "rh" when it has them,
        else those of the PFSS law the models here are trained on (r in
        [1, 2.5], drratio 2.5, nr = R + 2)."""
        z = np.load(path)
        Rs = int(z["grid"][2])
        g = grid_from_mesh(mesh)
        m = cls._from_saved(path, z, Grid(g.nth, g.nph, Rs, g.th, g.dth, g.ph, g.dph))
        if Rs != g.R:
            if "rh" in z:
                rh_s = np.asarray(z["rh"], np.float64)
            else:
                from .host import make_mesh
                rh_s = make_mesh(Rs + 2, 5, 8).rh
            m.set_radial(rh_s, mesh.rh, mesh.r[0], mesh.r[-1])
        return m

    def set_radial(self, rh_src, rh_dst, r0_dst, r1_dst):
        """Interpolation of the network's radial levels (half-mesh radii
        rh_src, ghosts included) onto the interior levels of rh_dst."""
        import torch
        idx, w = radial_weights(rh_src, rh_dst, r0_dst, r1_dst)
        self.R_out = len(idx)
        self.radial = (torch.tensor(idx).cuda(), torch.tensor(w, dtype=torch.float64).cuda())

    @classmethod
    def _from_saved(cls, path, z, grid: "Grid"):
        import torch
        _, _, _, W_, nl, mt, mp, hidden, in_ch = (int(v) for v in z["grid"])
        m = cls(grid, width=W_, layers=nl, mt=mt, mp=mp, hidden=hidden, in_ch=in_ch)
        for k in list(m.p):
            if "bf16_" + k in z:
                t = torch.from_numpy(z["bf16_" + k]).view(torch.bfloat16).to(torch.float32)
            else:
                t = torch.from_numpy(z["f32_" + k])
            if tuple(t.shape) != tuple(m.p[k].shape):
                raise ValueError(f"{path}: parameter {k} has shape {tuple(t.shape)}")
            m.p[k].copy_(t.cuda())
        m.pb = {k: v.to(torch.bfloat16).contiguous() for k, v in m.p.items() if v.dim() >= 2}
        return m

    def predict(self, x, sigma, out=None):
        """Initial guesses in the packed solver layout, FP64 [B, N] (into
        `out` when given); sigma: per-sample scales (host or FP64 device).
        With radial levels resampled (load_resampled) N counts the solver's
        levels."""
        import torch
        y = self.forward(x)  # FP32 [B, nph, nth, Rp]
        B = x.shape[0]
        g = self.g
        npos = g.nph * g.nth
        R = getattr(self, "R_out", g.R)
        assert y.dtype == torch.float32 and y.is_contiguous() and y.numel() == B * npos * self.Rp
        sig = sigma if hasattr(sigma, "data_ptr") else torch.tensor(np.asarray(sigma, np.float64), device="cuda")
        assert sig.dtype == torch.float64 and sig.numel() == B
        guess = out if out is not None else torch.empty((B, npos * R), dtype=torch.float64, device="cuda")
        if guess.dtype != torch.float64 or not guess.is_contiguous() or guess.numel() != B * npos * R:
            raise ValueError("predict: out must be a contiguous FP64 tensor of B x N")
        _count()
        if getattr(self, "radial", None) is not None:
            idx, w = self.radial
            _lib.check(_L().pot3d_fno_guess_resampled(
                C.c_void_p(y.data_ptr()), B, npos, self.Rp, g.R, C.c_void_p(idx.data_ptr()), C.c_void_p(w.data_ptr()),
                R, C.c_void_p(sig.data_ptr()), C.c_void_p(guess.data_ptr()), _stream()))
        else:
            _lib.check(_L().pot3d_fno_guess(C.c_void_p(y.data_ptr()), B, npos, self.Rp, g.R,
                                            C.c_void_p(sig.data_ptr()), C.c_void_p(guess.data_ptr()), _stream()))
        return guess


def _bf():
    import torch
    return torch.bfloat16
