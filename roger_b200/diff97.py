"""Differentiable 9/7 for rate-distortion training (no counterpart in the reference).

torch.autograd.Function bindings over the C ABI — the forward and inverse 9/7 DWT with their
hand-written adjoints as backward, the relaxed dead-zone quantiser (additive uniform noise of
one step per subband) with its backward, and the fused rate-distortion loss
    loss = mean((IDWT(Q(DWT(x))) - x)^2) + lam * sum_b sum log2(1 + |y_hat|/step_b)
differentiable with respect to the pixels x and the per-subband log steps.  torch provides the
device memory and the stream; every pass runs in libj2kb200's kernels.  The fused loss keeps three
planes per image for its backward: the quantiser input y, its noise u (so the backward does not
regenerate it) and the residual d = IDWT(y_hat) - x (the reconstruction itself is never stored;
the residual pass is fused into the last inverse level, and the "- 2/N d" term of the pixel
gradient into the last forward-adjoint level).  Where every level's width is a power of two in
64..1024, the quantiser runs inside the transforms: its forward as the forward levels write their
bands, y_hat as the inverse loads them (never stored), its backward as the transpose of the
inverse writes its bands.  The backward reads its output gradient on the device, so a step never
synchronises with the host.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib as L
from ._lib import check, lib
from .codec import default_context, subband_rects


def _parts(h):
    """Row ranges per image of the quantiser kernels (one partial sum per band and range)."""
    return max(1, min(int(h), 64))


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


def _band_sum(parts, n, nb, k):
    return parts.view(n, nb, k).sum(dim=2)


def relaxed_quant(y, log_steps, levels, seed, keep_noise=False):
    """-> (y_hat, rate per image and band (N, 3L+1)), plus the noise u when keep_noise."""
    ctx, h = _ctx(y)
    y = y.contiguous()
    n, hh, ww = y.shape
    nb, k = 3 * levels + 1, _parts(hh)
    ls = log_steps.detach().float().contiguous()
    yh = torch.empty_like(y)
    parts = torch.empty(n * nb * k, device=y.device, dtype=torch.float32)
    if keep_noise:
        u = torch.empty_like(y)
        check(lib().j2k_relaxed_quant_forward_noise(h, _p(y), _p(yh), _p(u), n, ww, hh, levels, _p(ls), seed,
                                                    _p(parts), k), h)
        return yh, _band_sum(parts, n, nb, k), u
    check(lib().j2k_relaxed_quant_forward(h, _p(y), _p(yh), n, ww, hh, levels, _p(ls), seed, _p(parts), k), h)
    return yh, _band_sum(parts, n, nb, k)


def relaxed_quant_backward(y, g_yhat, log_steps, levels, seed, lam, scale=None, alpha=1.0, noise=None):
    """-> (dL/dy, dL/dlog_steps) for L = <g, y_hat> + lam * sum(rate), g = scale * alpha * g_yhat
    (scale: optional 0-dim CUDA tensor, read on the device; noise: the forward's kept noise, else
    it is regenerated from seed)."""
    ctx, h = _ctx(y)
    n, hh, ww = y.shape
    nb, k = 3 * levels + 1, _parts(hh)
    ls = log_steps.detach().float().contiguous()
    gy = torch.empty_like(y)
    parts = torch.empty(n * nb * k, device=y.device, dtype=torch.float32)
    sp = None if scale is None else _p(scale)
    npt = None if noise is None else _p(noise.contiguous())
    check(lib().j2k_relaxed_quant_backward_scaled(h, _p(y.contiguous()), _p(g_yhat.contiguous()), _p(gy), n, ww, hh,
                                                  levels, _p(ls), seed, npt, float(lam), sp, float(alpha), _p(parts),
                                                  k), h)
    return gy, _band_sum(parts, n, nb, k).sum(dim=0)


def inverse_residual(y, x, levels):
    """-> (d = IDWT(y) - x, sum of d^2 as a 0-dim tensor), fused into the last inverse level."""
    ctx, h = _ctx(y)
    y, x = y.contiguous(), x.contiguous()
    n, hh, ww = y.shape
    d = torch.empty_like(y)
    parts = torch.empty(lib().j2k_dwt97_residual_partials(ww, hh, n), device=y.device, dtype=torch.float32)
    check(lib().j2k_dwt97_inverse_residual(h, _p(y), _p(x), _p(d), n, ww, hh, levels, _p(parts)), h)
    return d, parts.sum()


def forward_adjoint_residual(g, sub, levels, scale=None, alpha=1.0):
    """-> DWT^T(g) - scale * alpha * sub, fused into the last adjoint level."""
    ctx, h = _ctx(g)
    g, sub = g.contiguous(), sub.contiguous()
    n, hh, ww = g.shape
    out = torch.empty_like(g)
    sp = None if scale is None else _p(scale)
    check(lib().j2k_dwt97_forward_adjoint_residual(h, _p(g), _p(sub), sp, float(alpha), _p(out), n, ww, hh, levels),
          h)
    return out


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


def _rd_forward(x, log_steps, levels, lam, seed):
    """The forward of the fused loss (j2k_dwt97_rd_forward): y = DWT(x) with the quantiser's
    noise u drawn as each level writes its bands, the residual d = IDWT(y_hat) - x with y_hat
    formed as the inverse loads the bands, and the loss scalar from the partial sums.  Returns
    (loss, y, d, u)."""
    x = x.detach().contiguous()
    c, h = _ctx(x)
    n, hh, ww = x.shape
    nb, kp = 3 * levels + 1, lib().j2k_dwt97_rd_parts(h, ww, hh, levels)
    ls = log_steps.detach().float().contiguous()
    y, u, d = torch.empty_like(x), torch.empty_like(x), torch.empty_like(x)
    rparts = torch.empty(n * nb * kp, device=x.device, dtype=torch.float32)
    sparts = torch.empty(lib().j2k_dwt97_residual_partials(ww, hh, n), device=x.device, dtype=torch.float32)
    check(lib().j2k_dwt97_rd_forward(h, _p(x), _p(y), _p(u), _p(d), n, ww, hh, levels, _p(ls), seed, _p(rparts),
                                     _p(sparts)), h)
    # the loss scalar from both sets of partial sums, in one launch
    loss = torch.empty((), device=x.device, dtype=torch.float32)
    check(lib().j2k_dwt97_rd_finalize(h, _p(rparts), rparts.numel(), _p(sparts), sparts.numel(),
                                      1.0 / x.numel(), float(lam), _p(loss)), h)
    return loss, y, d, u


def _rd_backward(y, d, u, log_steps, g, levels, lam, seed):
    """The backward of the fused loss for output gradient g (0-dim, read on the device),
    j2k_dwt97_rd_backward: the transpose of the inverse applied to the residual with the
    quantiser backward (scaled by 2/N and g) in its band writes, then the transpose of the
    forward with the -2/N residual term; the per-band log-step gradient in one launch.
    Returns (dL/dx, dL/dlog_steps)."""
    del seed  # the backward reads the forward's noise u
    g = g.detach().float().contiguous()
    c, h = _ctx(y)
    n, hh, ww = y.shape
    nb, kp = 3 * levels + 1, lib().j2k_dwt97_rd_parts(h, ww, hh, levels)
    ls = log_steps.detach().float().contiguous()
    g_y, gx = torch.empty_like(y), torch.empty_like(y)
    parts = torch.empty(n * nb * kp, device=y.device, dtype=torch.float32)
    check(lib().j2k_dwt97_rd_backward(h, _p(y), _p(u), _p(d), _p(ls), float(lam), _p(g), 2.0 / d.numel(), _p(g_y),
                                      _p(gx), n, ww, hh, levels, _p(parts)), h)
    del g_y
    g_ls = torch.empty(nb, device=y.device, dtype=torch.float32)  # per band, in one launch
    check(lib().j2k_dwt97_band_sum(h, _p(parts), n, nb, kp, _p(g_ls)), h)
    return gx, g_ls


class RDLoss(torch.autograd.Function):
    """Fused rate-distortion loss of a (N, H, W) float32 batch (one 0-dim CUDA tensor).
    Forward: DWT, quantiser, inverse with the residual fused in.  Backward: inverse adjoint of
    the residual, quantiser backward (scaled by 2/N and the output gradient on the device),
    forward adjoint with the -2/N residual fused in.

    checkpoint=True keeps nothing of the forward for the backward but the input: the lifting
    outputs of every level (the coefficients y), the quantiser's noise and the residual are
    recomputed in the backward from x (one more forward DWT, quantiser and inverse).  Between
    the two passes the step then holds x alone instead of x, y, u and d, which is what lets a
    batch, or one image, that does not fit four times over run at all; the gradients are
    identical to the stored form's (the recomputation is the same deterministic kernels, the
    noise the same Philox counters)."""

    @staticmethod
    def forward(ctx, x, log_steps, levels, lam, seed, checkpoint=False):
        loss, y, d, u = _rd_forward(x, log_steps, levels, lam, seed)
        if checkpoint:
            del y, d, u
            ctx.save_for_backward(x, log_steps)
        else:
            ctx.save_for_backward(y, d, u, log_steps)
        ctx.levels, ctx.lam, ctx.seed, ctx.checkpoint = levels, lam, seed, checkpoint
        return loss

    @staticmethod
    def backward(ctx, g):
        if ctx.checkpoint:
            x, log_steps = ctx.saved_tensors
            _, y, d, u = _rd_forward(x, log_steps, ctx.levels, ctx.lam, ctx.seed)
        else:
            y, d, u, log_steps = ctx.saved_tensors
        gx, g_ls = _rd_backward(y, d, u, log_steps, g, ctx.levels, ctx.lam, ctx.seed)
        return gx, g_ls.to(log_steps.dtype), None, None, None, None


def rd_loss(x, log_steps, levels=5, lam=0.01, seed=0, checkpoint=False):
    """Rate-distortion loss of a (N, H, W) float32 batch; differentiable in x and log_steps.
    checkpoint=True recomputes the forward's intermediates in the backward instead of keeping
    them (see RDLoss)."""
    return RDLoss.apply(x, log_steps, levels, lam, seed, checkpoint)


def rd_loss_composed(x, log_steps, levels=5, lam=0.01, seed=0):
    """The same loss composed from the separate autograd pieces (DWT97, RelaxedQuant, IDWT97
    and torch's MSE); kept to check the fused form against."""
    y = DWT97.apply(x, levels)
    yh, rate = RelaxedQuant.apply(y, log_steps, levels, seed)
    xh = IDWT97.apply(yh, levels)
    return torch.mean((xh - x) ** 2) + lam * rate.sum()


def rd_loss_and_grads(x, log_steps, levels=5, lam=0.01, seed=0, chunk=None):
    """Loss and gradients computed chunk by chunk (images [i, i+chunk) at a time), so the peak
    device memory is that of one chunk (its coefficients and residual) when the whole batch
    does not fit in HBM.  Returns (loss as a 0-dim tensor, dL/dx, dL/dlog_steps)."""
    n = x.shape[0]
    chunk = chunk or n
    total = float(x.numel())
    alpha = 2.0 / total
    gx = torch.empty_like(x)
    gls = torch.zeros_like(log_steps, dtype=torch.float32)
    loss = torch.zeros((), device=x.device, dtype=torch.float32)
    for i in range(0, n, chunk):
        xc = x[i:i + chunk].contiguous()
        y = dwt97(xc, levels)
        yh, rate = relaxed_quant(y, log_steps, levels, seed + i)
        d, sq = inverse_residual(yh, xc, levels)
        del yh
        loss += sq / total + lam * rate.sum()
        g_res = idwt97_adjoint(d, levels)
        g_y, g_ls = relaxed_quant_backward(y, g_res, log_steps, levels, seed + i, lam, alpha=alpha)
        del g_res, y
        gx[i:i + chunk] = forward_adjoint_residual(g_y, d, levels, alpha=alpha)
        gls += g_ls
    return loss, gx, gls


class GraphedRDStep:
    """One rate-distortion step (loss, its gradient with respect to the pixels and the log-steps)
    captured once in a CUDA graph and replayed: a step is then one graph launch, with no
    per-kernel host work.  The inputs are static: write new pixels or log-steps into `x` and
    `log_steps` (in place) before calling; the results are the tensors `loss`, `x.grad` and
    `log_steps.grad`, overwritten by every call.  Capture warms up first (library scratch,
    autograd) on a side stream, as CUDA-graph capture requires."""

    def __init__(self, x, log_steps, levels=5, lam=0.01, seed=0, warmup=3):
        if not (x.is_cuda and x.requires_grad and log_steps.requires_grad):
            raise ValueError("GraphedRDStep: x and log_steps must be CUDA tensors that require grad")
        self.x, self.log_steps = x, log_steps
        args = (levels, lam, seed)
        side = torch.cuda.Stream(device=x.device)
        side.wait_stream(torch.cuda.current_stream(x.device))
        with torch.cuda.stream(side):
            for _ in range(warmup):
                x.grad = None
                log_steps.grad = None
                rd_loss(x, log_steps, *args).backward()
        torch.cuda.current_stream(x.device).wait_stream(side)
        x.grad = None
        log_steps.grad = None
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.loss = rd_loss(x, log_steps, *args)
            self.loss.backward()

    def __call__(self):
        self.graph.replay()
        return self.loss
