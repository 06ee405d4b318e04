"""GPU tests of the differentiable 9/7 path: adjoint kernels against the FP64 oracle's adjoints
and against explicit transposes, the rate-distortion gradient against FP64 finite differences
of the oracle (config 3 setting on a 64x64 crop), and the chunked (memory-bounded) form
against the one-shot autograd form."""
import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from roger_b200 import synth

pytestmark = pytest.mark.gpu
ADJ_TOL = 1e-5   # FP32 adjoint vs FP64 oracle, relative to the largest magnitude
GRAD_TOL = 1e-4  # FP32 analytic gradient vs FP64 finite differences (h = 1e-6), relative


@pytest.fixture(scope="module")
def D():
    from roger_b200 import diff97
    return diff97


@pytest.mark.parametrize("w,h,L", [(77, 53, 3), (64, 64, 5), (1, 9, 2), (33, 2, 3), (128, 96, 5), (700, 90, 3),
                                   (517, 35, 4), (1024, 40, 2), (8, 2, 1), (250, 300, 5)])
def test_adjoints_match_fp64_oracle(D, w, h, L):
    rng = np.random.default_rng(w * h + L)
    g = rng.normal(size=(2, h, w))
    gt = torch.from_numpy(g.astype(np.float32)).cuda()
    fa = D.dwt97_adjoint(gt, L).cpu().numpy()
    ia = D.idwt97_adjoint(gt, L).cpu().numpy()
    for i in range(2):
        rf = O.dwt97_fwd_adj(g[i], L)
        ri = O.dwt97_inv_adj(g[i], L)
        assert np.abs(fa[i] - rf).max() <= ADJ_TOL * np.abs(rf).max()
        assert np.abs(ia[i] - ri).max() <= ADJ_TOL * np.abs(ri).max()


@pytest.mark.parametrize("w,h,L", [(9, 7, 2), (16, 16, 3), (6, 11, 2)])
def test_adjoints_are_explicit_transposes(D, w, h, L):
    n = w * h
    eye = torch.eye(n, device="cuda", dtype=torch.float32).view(n, h, w)
    F = D.dwt97(eye, L).view(n, n).T.cpu().double().numpy()        # F[:, i] = DWT(e_i)
    Finv = D.idwt97(eye, L).view(n, n).T.cpu().double().numpy()
    Fa = D.dwt97_adjoint(eye, L).view(n, n).T.cpu().double().numpy()
    Ia = D.idwt97_adjoint(eye, L).view(n, n).T.cpu().double().numpy()
    assert np.abs(Fa - F.T).max() <= 1e-5
    assert np.abs(Ia - Finv.T).max() <= 1e-5
    # and the FP64 oracle's explicit transpose
    F64 = np.stack([O.dwt97_fwd(np.eye(n)[i].reshape(h, w), L, f64=True).ravel() for i in range(n)], 1)
    assert np.abs(Fa - F64.T).max() <= 1e-5


def _crop():
    x = synth.gray(1024, 1024, 200)[:64, :64].astype(np.float64) / 255.0
    return x


def test_rd_loss_and_gradients_match_fp64_finite_differences(D):
    L, lam, seed = 5, 0.01, 200
    x = _crop()
    ls = np.full(3 * L + 1, math.log(1 / 64.0))
    xt = torch.from_numpy(x.astype(np.float32))[None].cuda().requires_grad_(True)
    lt = torch.from_numpy(ls.astype(np.float32)).cuda().requires_grad_(True)
    loss = D.rd_loss(xt, lt, L, lam, seed)
    loss.backward()
    gx = xt.grad[0].cpu().double().numpy()
    gl = lt.grad.cpu().double().numpy()
    ref_loss, ref_gx, ref_gl = O.rd_loss(x, L, ls, lam, seed)
    assert abs(loss.item() - ref_loss) <= 1e-5 * abs(ref_loss)
    # analytic FP64 gradients of the oracle are the FD-checked reference (tests/test_oracle.py);
    # here the GPU gradients are compared with FD64 directly on sampled pixels and every step
    h = 1e-6
    rng = np.random.default_rng(1)
    scale_x = np.abs(ref_gx).max()
    for _ in range(24):
        i, j = rng.integers(0, 64, 2)
        xp, xm = x.copy(), x.copy()
        xp[i, j] += h
        xm[i, j] -= h
        fd = (O.rd_loss(xp, L, ls, lam, seed, False) - O.rd_loss(xm, L, ls, lam, seed, False)) / (2 * h)
        assert abs(gx[i, j] - fd) <= GRAD_TOL * max(abs(fd), 0.05 * scale_x), (i, j, gx[i, j], fd)
    for b in range(len(ls)):
        lp, lm = ls.copy(), ls.copy()
        lp[b] += h
        lm[b] -= h
        fd = (O.rd_loss(x, L, lp, lam, seed, False) - O.rd_loss(x, L, lm, lam, seed, False)) / (2 * h)
        assert abs(gl[b] - fd) <= GRAD_TOL * max(abs(fd), 1e-3), (b, gl[b], fd)
    assert np.abs(gx - ref_gx).max() <= 1e-4 * scale_x


def test_chunked_form_matches_autograd(D):
    L, lam, seed = 4, 0.01, 7
    xs = np.stack([synth.gray(96, 80, 300 + k) for k in range(4)]).astype(np.float32) / 255.0
    xt = torch.from_numpy(xs).cuda().requires_grad_(True)
    lt = torch.full((3 * L + 1,), math.log(1 / 64.0), device="cuda", requires_grad=True)
    loss = D.rd_loss(xt, lt, L, lam, seed)
    loss.backward()
    l2, gx2, gl2 = D.rd_loss_and_grads(xt.detach(), lt.detach(), L, lam, seed, chunk=1)
    assert abs(loss.item() - float(l2)) <= 1e-5 * abs(float(l2))
    assert torch.allclose(xt.grad, gx2, rtol=1e-4, atol=1e-7)
    assert torch.allclose(lt.grad, gl2, rtol=1e-4, atol=1e-6)


@pytest.mark.parametrize("w,h,L", [(37, 29, 3), (64, 48, 2), (5, 3, 1)])
def test_relaxed_quantiser_matches_oracle_noise(D, w, h, L):
    """y_hat = (y/step + u) * step with u drawn as the oracle draws it (one Philox4x32-10 block
    per 4 samples of a plane row); per-band rates against an FP64 sum."""
    rng = np.random.default_rng(w + h)
    n, seed = 2, 77
    y = rng.normal(scale=20.0, size=(n, h, w)).astype(np.float32)
    ls = np.linspace(-1.0, 2.0, 3 * L + 1).astype(np.float32)
    yh, rate = D.relaxed_quant(torch.from_numpy(y).cuda(), torch.from_numpy(ls).cuda(), L, seed)
    yh, rate = yh.cpu().numpy(), rate.cpu().numpy()
    bands = O.subbands(w, h, L)
    for i in range(n):
        ref = np.zeros((h, w))
        rref = np.zeros(3 * L + 1)
        for b, (bx, by, bw, bh, _o, _l) in enumerate(bands):
            st = float(np.exp(np.float64(ls[b])))
            for yy in range(by, by + bh):
                for xx in range(bx, bx + bw):
                    t = y[i, yy, xx] / st + O.rd_noise(seed + i, w, xx, yy)
                    ref[yy, xx] = t * st
                    rref[b] += np.log2(1.0 + abs(t))
        assert np.abs(yh[i] - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max())
        assert np.allclose(rate[i], rref, rtol=1e-4, atol=1e-3)


@pytest.mark.parametrize("n,w,h,L", [(3, 300, 70, 4), (2, 64, 64, 5), (1, 9, 5, 2)])
def test_fused_rd_loss_matches_composed_form(D, n, w, h, L):
    """The fused loss (residual fused into the inverse and into the forward adjoint, output
    gradient read on the device) against the same loss composed from the separate pieces."""
    x = torch.from_numpy(synth.float_batch(n, w, h, 40)).cuda()
    ls = torch.linspace(-4.0, -2.0, 3 * L + 1, device="cuda")
    x1, l1 = x.clone().requires_grad_(True), ls.clone().requires_grad_(True)
    x2, l2 = x.clone().requires_grad_(True), ls.clone().requires_grad_(True)
    a = D.rd_loss(x1, l1, L, 0.01, 9)
    b = D.rd_loss_composed(x2, l2, L, 0.01, 9)
    (3.0 * a).backward()
    (3.0 * b).backward()
    assert abs(a.item() - b.item()) <= 1e-5 * abs(b.item())
    assert torch.allclose(x1.grad, x2.grad, rtol=1e-3, atol=1e-7 * x2.grad.abs().max().item())
    assert torch.allclose(l1.grad, l2.grad, rtol=1e-4, atol=1e-6)


def test_kept_noise_matches_regenerated_noise(D):
    """The forward that keeps its noise writes exactly the oracle's noise, and the backward that
    reads it gives the same gradients as the backward that regenerates it."""
    n, w, h, L, seed = 2, 70, 37, 3, 5
    rng = np.random.default_rng(3)
    y = torch.from_numpy(rng.normal(scale=10.0, size=(n, h, w)).astype(np.float32)).cuda()
    ls = torch.linspace(-1.0, 1.0, 3 * L + 1, device="cuda")
    yh, rate, u = D.relaxed_quant(y, ls, L, seed, keep_noise=True)
    yh2, rate2 = D.relaxed_quant(y, ls, L, seed)
    assert torch.equal(yh, yh2) and torch.equal(rate, rate2)
    un = u.cpu().numpy()
    for i in range(n):
        for yy, xx in [(0, 0), (5, 3), (36, 69), (17, 40)]:
            assert un[i, yy, xx] == np.float32(O.rd_noise(seed + i, w, xx, yy))
    g = torch.from_numpy(rng.normal(size=(n, h, w)).astype(np.float32)).cuda()
    a = D.relaxed_quant_backward(y, g, ls, L, seed, 0.01, noise=u)
    b = D.relaxed_quant_backward(y, g, ls, L, seed, 0.01)
    assert torch.equal(a[0], b[0]) and torch.allclose(a[1], b[1], rtol=1e-6, atol=0)


def test_graphed_step_matches_eager_step(D):
    """The CUDA-graph replay of a step gives the eager step's loss and gradients exactly, and
    follows new inputs written into its static tensors."""
    L = 3
    x = torch.from_numpy(synth.float_batch(2, 96, 80, 60)).cuda().requires_grad_(True)
    ls = torch.full((3 * L + 1,), -4.0, device="cuda", requires_grad=True)
    step = D.GraphedRDStep(x, ls, L, 0.01, 7)
    for k in range(2):
        with torch.no_grad():
            x.mul_(0.5 + 0.25 * k)
        loss = step().item()
        xe = x.detach().clone().requires_grad_(True)
        le = ls.detach().clone().requires_grad_(True)
        ref = D.rd_loss(xe, le, L, 0.01, 7)
        ref.backward()
        assert loss == ref.item()
        assert torch.equal(x.grad, xe.grad) and torch.equal(ls.grad, le.grad)


def test_checkpointed_step_matches_stored_step_and_fd64(D):
    """checkpoint=True (the forward keeps only x; the backward recomputes the coefficients,
    the noise and the residual) gives the stored form's loss and gradients exactly, holds less
    memory between the passes, and matches FP64 finite differences on the config's crop."""
    L, lam, seed = 5, 0.01, 200
    xs = torch.from_numpy(synth.float_batch(3, 256, 192, 70)).cuda()
    ls0 = torch.full((3 * L + 1,), math.log(1 / 64.0), device="cuda")
    res = []
    for ck in (False, True):
        x = xs.clone().requires_grad_(True)
        ls = ls0.clone().requires_grad_(True)
        torch.cuda.synchronize()
        base = torch.cuda.memory_allocated()
        loss = D.rd_loss(x, ls, L, lam, seed, checkpoint=ck)
        held = torch.cuda.memory_allocated() - base  # kept for the backward
        loss.backward()
        res.append((loss.item(), x.grad.clone(), ls.grad.clone(), held))
    assert res[0][0] == res[1][0]
    assert torch.equal(res[0][1], res[1][1]) and torch.equal(res[0][2], res[1][2])
    plane = xs.numel() * 4
    assert res[0][3] >= 3 * plane and res[1][3] < plane  # y, d and u kept, against none
    # FD64 on the 64x64 crop of config 3, checkpointed
    x = _crop()
    lsn = np.full(3 * L + 1, math.log(1 / 64.0))
    xt = torch.from_numpy(x.astype(np.float32))[None].cuda().requires_grad_(True)
    lt = torch.from_numpy(lsn.astype(np.float32)).cuda().requires_grad_(True)
    D.rd_loss(xt, lt, L, lam, seed, checkpoint=True).backward()
    gx = xt.grad[0].cpu().double().numpy()
    gl = lt.grad.cpu().double().numpy()
    h = 1e-6
    _, ref_gx, _ = O.rd_loss(x, L, lsn, lam, seed)
    scale_x = np.abs(ref_gx).max()
    rng = np.random.default_rng(5)
    for _ in range(12):
        i, j = rng.integers(0, 64, 2)
        xp, xm = x.copy(), x.copy()
        xp[i, j] += h
        xm[i, j] -= h
        fd = (O.rd_loss(xp, L, lsn, lam, seed, False) - O.rd_loss(xm, L, lsn, lam, seed, False)) / (2 * h)
        assert abs(gx[i, j] - fd) <= GRAD_TOL * max(abs(fd), 0.05 * scale_x)
    for b in range(0, len(lsn), 3):
        lp, lm = lsn.copy(), lsn.copy()
        lp[b] += h
        lm[b] -= h
        fd = (O.rd_loss(x, L, lp, lam, seed, False) - O.rd_loss(x, L, lm, lam, seed, False)) / (2 * h)
        assert abs(gl[b] - fd) <= GRAD_TOL * max(abs(fd), 1e-3)


# ---- band kernels (levels 64..1024 wide as full-row bands) against the strip kernels ----------

def _rows(on):
    """Switch the default context between the band kernels (on) and the strip kernels."""
    from roger_b200._lib import lib
    from roger_b200.codec import default_context
    assert lib().j2k_ctx_set_tuning(default_context(0).h, 13, 1 if on else 0) == 0


def _both(fn):
    _rows(False)
    try:
        a = fn()
    finally:
        _rows(True)
    return a, fn()


BAND_SHAPES = [(2, 1024, 64, 5), (2, 512, 96, 4), (1, 256, 37, 3), (3, 64, 40, 1), (1, 128, 2, 1),
               (1, 1024, 80, 6), (2, 256, 256, 3)]


@pytest.mark.parametrize("n,w,h,L", BAND_SHAPES)
def test_band_kernels_bit_identical_to_strip_kernels(D, n, w, h, L):
    """Both adjoints and the inverse with its residual, per level through the band kernels where
    the level width allows (1024 x 80 at L=6: the 32-wide level runs as a strip-kernel
    sub-transform), equal the strip kernels bit for bit; the residual's partial sums add up to
    the same total."""
    g = torch.from_numpy(np.random.default_rng(w + h + L).normal(size=(n, h, w)).astype(np.float32)).cuda()
    x = torch.from_numpy(np.random.default_rng(7 * w + h).normal(size=(n, h, w)).astype(np.float32)).cuda()
    fa0, fa1 = _both(lambda: D.dwt97_adjoint(g, L))
    ia0, ia1 = _both(lambda: D.idwt97_adjoint(g, L))
    assert torch.equal(fa0, fa1)
    assert torch.equal(ia0, ia1)
    (d0, s0), (d1, s1) = _both(lambda: D.inverse_residual(g, x, L))
    assert torch.equal(d0, d1)
    assert abs(s0.item() - s1.item()) <= 1e-5 * abs(s0.item())
    gsc = torch.tensor(1.7, device="cuda")
    r0, r1 = _both(lambda: D.forward_adjoint_residual(g, x, L, scale=gsc, alpha=0.3))
    assert torch.equal(r0, r1)


@pytest.mark.parametrize("n,w,h,L", [(2, 1024, 64, 5), (1, 512, 50, 4), (2, 128, 128, 2), (1, 64, 64, 1),
                                     (1, 1024, 80, 6)])
def test_fused_rd_step_matches_separate_passes(D, n, w, h, L):
    """The fused step (quantiser inside the band kernels) against the separate passes of the strip
    kernels: y, u, d and dL/dx bit for bit (the same operations per sample), the loss and the
    log-step gradient to 1e-5 (their partial sums are added in another order)."""
    lam, seed = 0.01, 11
    x = torch.from_numpy(np.stack([synth.gray(w, h, 300 + i) for i in range(n)]).astype(np.float32) / 255).cuda()
    ls = torch.full((3 * L + 1,), math.log(1 / 64.0), device="cuda")
    ls += torch.linspace(-0.3, 0.3, 3 * L + 1, device="cuda")

    def step():
        loss, y, d, u = D._rd_forward(x, ls, L, lam, seed)
        gx, gl = D._rd_backward(y, d, u, ls, torch.tensor(1.5, device="cuda"), L, lam, seed)
        return [t.clone() for t in (loss, y, d, u, gx, gl)]

    a, b = _both(step)
    for i in (1, 2, 3, 4):
        assert torch.equal(a[i], b[i]), i
    assert abs(a[0].item() - b[0].item()) <= 1e-5 * abs(a[0].item())
    assert torch.allclose(a[5], b[5], rtol=1e-5, atol=1e-7 * a[5].abs().max().item())
