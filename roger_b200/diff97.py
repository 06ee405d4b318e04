"""Differentiable 9/7 for rate-distortion training (no counterpart in the reference).

Three torch.autograd.Function bindings over the C ABI — the forward and inverse 9/7 DWT with
their hand-written adjoints as backward, and the relaxed dead-zone quantiser (additive uniform
noise of one step per subband) with its backward — and the loss they compose:
    loss = mean((IDWT(Q(DWT(x))) - x)^2) + lam * sum_b sum log2(1 + |y_hat|/step_b)
differentiable with respect to the pixels x and the per-subband log steps.  torch provides the
device memory, the stream and the elementwise MSE; the transforms, adjoints and quantiser run
in libj2kb200's kernels.  No lifting intermediate is kept: the DWT is linear, so its backward
needs only the incoming gradient; the quantiser keeps its input y (or recomputes it from x in
the chunked form, which bounds memory when the batch does not fit in HBM).
"""
import ctypes as C

import numpy as np
import torch

from . import _lib as L
from ._lib import check, lib
from .codec import default_context, subband_rects

PARTS = 64  # partial sums per (image, band)


def _p(t):
    return C.c_void_p(t.data_ptr())


def _ctx(t):
    ctx = default_context(t.device.index or 0)
    return ctx, ctx._bind()


def dwt97(x, levels):
    """Forward 9/7 (T.800 order) of a (N, H, W) float32 CUDA batch -> Mallat planes."""
    ctx, h = _ctx(x)
    x = x.contiguous()
    n, hh, ww = x.shape
    y = torch.empty_like(x)
    check(lib().j2k_dwt_forward_batch(h, L.W97, L.ORDER_T800, _p(x), ww, ww * hh, _p(y), ww, ww * hh, n, ww, hh,
                                      levels, None), h)
    return y


def idwt97(y, levels):
    ctx, h = _ctx(y)
    y = y.contiguous()
    n, hh, ww = y.shape
    x = torch.empty_like(y)
    check(lib().j2k_dwt_inverse_batch(h, L.W97, L.ORDER_T800, _p(y), ww, ww * hh, _p(x), ww, ww * hh, n, ww, hh,
                                      levels, None), h)
    return x


def dwt97_adjoint(g, levels):
    ctx, h = _ctx(g)
    g = g.contiguous()
    n, hh, ww = g.shape
    out = torch.empty_like(g)
    check(lib().j2k_dwt97_forward_adjoint(h, _p(g), _p(out), n, ww, hh, levels), h)
    return out


def idwt97_adjoint(g, levels):
    ctx, h = _ctx(g)
    g = g.contiguous()
    n, hh, ww = g.shape
    out = torch.empty_like(g)
    check(lib().j2k_dwt97_inverse_adjoint(h, _p(g), _p(out), n, ww, hh, levels), h)
    return out


def _band_sum(parts, n, nb):
    return parts.view(n, nb, PARTS).sum(dim=2)


def relaxed_quant(y, log_steps, levels, seed):
    """-> (y_hat, rate per image and band (N, 3L+1))."""
    ctx, h = _ctx(y)
    y = y.contiguous()
    n, hh, ww = y.shape
    nb = 3 * levels + 1
    ls = log_steps.detach().float().contiguous()
    yh = torch.empty_like(y)
    parts = torch.empty(n * nb * PARTS, device=y.device, dtype=torch.float32)
    check(lib().j2k_relaxed_quant_forward(h, _p(y), _p(yh), n, ww, hh, levels, _p(ls), seed, _p(parts), PARTS), h)
    return yh, _band_sum(parts, n, nb)


def relaxed_quant_backward(y, g_yhat, log_steps, levels, seed, lam):
    ctx, h = _ctx(y)
    n, hh, ww = y.shape
    nb = 3 * levels + 1
    ls = log_steps.detach().float().contiguous()
    gy = torch.empty_like(y)
    parts = torch.empty(n * nb * PARTS, device=y.device, dtype=torch.float32)
    check(lib().j2k_relaxed_quant_backward(h, _p(y.contiguous()), _p(g_yhat.contiguous()), _p(gy), n, ww, hh,
                                           levels, _p(ls), seed, float(lam), _p(parts), PARTS), h)
    return gy, _band_sum(parts, n, nb).sum(dim=0)


class DWT97(torch.autograd.Function):
    """y = DWT(x); backward applies the hand-written forward adjoint."""

    @staticmethod
    def forward(ctx, x, levels):
        ctx.levels = levels
        return dwt97(x, levels)

    @staticmethod
    def backward(ctx, g):
        return dwt97_adjoint(g, ctx.levels), None


class IDWT97(torch.autograd.Function):
    """x = IDWT(y); backward applies the hand-written inverse adjoint."""

    @staticmethod
    def forward(ctx, y, levels):
        ctx.levels = levels
        return idwt97(y, levels)

    @staticmethod
    def backward(ctx, g):
        return idwt97_adjoint(g, ctx.levels), None


class RelaxedQuant(torch.autograd.Function):
    """(y_hat, rate) = Q(y, log_steps).  The rate gradient must be the same scalar weight for
    every image and band (the loss weights sum(rate) by lam)."""

    @staticmethod
    def forward(ctx, y, log_steps, levels, seed):
        yh, rate = relaxed_quant(y, log_steps, levels, seed)
        ctx.save_for_backward(y, log_steps)
        ctx.levels, ctx.seed = levels, seed
        return yh, rate

    @staticmethod
    def backward(ctx, g_yhat, g_rate):
        y, log_steps = ctx.saved_tensors
        if g_rate is None:
            lam = 0.0
        else:
            lam = float(g_rate.flatten()[0])
            if not torch.allclose(g_rate, torch.full_like(g_rate, lam)):
                raise ValueError("RelaxedQuant: rate gradient must be uniform (loss = ... + lam * rate.sum())")
        if g_yhat is None:
            g_yhat = torch.zeros_like(y)
        gy, gls = relaxed_quant_backward(y, g_yhat, log_steps, ctx.levels, ctx.seed, lam)
        return gy, gls.to(log_steps.dtype), None, None


def rd_loss(x, log_steps, levels=5, lam=0.01, seed=0):
    """Rate-distortion loss of a (N, H, W) float32 batch; differentiable in x and log_steps."""
    y = DWT97.apply(x, levels)
    yh, rate = RelaxedQuant.apply(y, log_steps, levels, seed)
    xh = IDWT97.apply(yh, levels)
    return torch.mean((xh - x) ** 2) + lam * rate.sum()


def rd_loss_and_grads(x, log_steps, levels=5, lam=0.01, seed=0, chunk=None):
    """Loss and gradients computed chunk by chunk (images [i, i+chunk) at a time), so the peak
    device memory is that of one chunk: the quantiser input is recomputed from the chunk's
    pixels in the backward instead of being kept for the whole batch."""
    n = x.shape[0]
    chunk = chunk or n
    total = float(x.numel())
    gx = torch.empty_like(x)
    gls = torch.zeros_like(log_steps, dtype=torch.float32)
    loss = 0.0
    for i in range(0, n, chunk):
        xc = x[i:i + chunk].contiguous()
        # forward
        y = dwt97(xc, levels)
        yh, rate = relaxed_quant(y, log_steps, levels, seed + i)
        del y
        xh = idwt97(yh, levels)
        del yh
        d = xh - xc
        loss += float((d * d).sum()) / total + lam * float(rate.sum())
        # backward (recompute y from the chunk's pixels)
        g_xh = (2.0 / total) * d
        g_yh = idwt97_adjoint(g_xh, levels)
        y = dwt97(xc, levels)
        g_y, g_ls = relaxed_quant_backward(y, g_yh, log_steps, levels, seed + i, lam)
        gx[i:i + chunk] = dwt97_adjoint(g_y, levels) - g_xh
        gls += g_ls
    return loss, gx, gls
