"""CPU FP32 autograd restatement of pot3d_b200.fno.FNO -- TEST INFRASTRUCTURE.

Same bases, same (BF16-rounded) weights, same layer sequence, evaluated with
torch on the CPU in FP32; its loss and parameter gradients are the reference
for the GPU forward/backward kernels.
"""
import math

import numpy as np
import torch


def reference_loss_and_grads(model, x_bf16, target):
    """model: pot3d_b200.fno.FNO (its weights are read back to the CPU).
    x_bf16: [B, nph, nth, 64] inputs; target: [B, nph, nth, R] FP32."""
    g = model.g
    W_, mt, mp = model.W, model.mt, model.mp
    P = {k: v.detach().cpu().to(torch.bfloat16).float().requires_grad_(True) for k, v in model.p.items()}
    Ft = model.Ft.cpu().float()[:, :g.nth]
    Fp = model.Fp.cpu().float()[:, :g.nph]
    Gt = model.Gt.cpu().float()[:g.nth, :mt]
    Gp = model.Gp.cpu().float()[:g.nph, :mp]
    x = x_bf16.cpu().float()[..., :model.in_ch]
    B = x.shape[0]
    gelu = lambda t: 0.5 * t * (1 + torch.tanh(0.7978845608028654 * (t + 0.044715 * t ** 3)))
    v = x @ P["Plift"][:, :model.in_ch].T + P["blift"]
    for l in range(model.nl):
        # spectral: [B, nph, nth, W] -> modes [B, W, mt, mp]
        vt = v.permute(0, 3, 1, 2)  # [B, W, nph, nth]
        c1 = torch.einsum("bckj,mj->bckm", vt, Ft)       # theta analysis
        c2 = torch.einsum("bckm,nk->bcmn", c1, Fp)       # phi analysis
        R = P[f"R{l}"][:, :, :W_].view(mt, mp, W_, W_)   # [mt, mp, c', c]
        c3 = torch.einsum("bcmn,mnec->bemn", c2, R)      # per-mode channel mixing
        s1 = torch.einsum("bemn,kn->bemk", c3, Gp)       # phi synthesis
        s2 = torch.einsum("bemk,jm->bekj", s1, Gt)       # theta synthesis
        spec = s2.permute(0, 2, 3, 1)                    # [B, nph, nth, W]
        pre = v @ P[f"W{l}"][:, :W_].T + P[f"b{l}"] + spec
        v = pre if l == model.nl - 1 else gelu(pre)
    h = gelu(v @ P["Q1"][:, :W_].T + P["bq1"])
    out = h @ P["Q2"][:g.R, :].T + P["bq2"][:g.R]
    t = target.cpu().float()
    num = ((out - t) ** 2).sum(dim=(1, 2, 3))
    den = (t ** 2).sum(dim=(1, 2, 3))
    loss = (num / den).mean()
    loss.backward()
    return loss.item(), {k: v.grad for k, v in P.items()}
