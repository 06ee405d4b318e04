"""GPU parity at the benchmark configurations' full sizes, against the CPU oracle.

The other parity tests run at 512x512 and below.  These run the workloads themselves:
  * 4096x4096 RGB lossless (RCT + 5/3, 6 levels, 64x64 code-blocks): the codestream, hence every
    one of the 12,288 code-blocks' codewords, byte-equal to the oracle's, and its decode equal
    to the input;
  * 4096x4096 RGB lossy (ICT + 9/7 FP32, 6 levels, steps 8*2^-k): the quantised indices and the
    codestream equal to the oracle's, and the decode equal to the oracle's reconstruction;
  * the 256-image mixed set (log-uniform sizes in [64, 2048], 5/3 and 9/7, gray and RGB, 3-5
    levels, 32x32 and 64x64 code-blocks) through the batched encoder: every image's codestream
    equal to the oracle's; and through the batched decoder: 5/3 images exact, 9/7 images equal
    to the oracle's reconstruction;
  * 16 x 1024x1024 float32, 9/7 with 5 levels: forward and inverse bit-identical to the FP32
    oracle, the error per subband against the FP64 oracle, and one rate-distortion step's loss
    and gradients against the FP64 oracle's.
The oracle encodes run on a pool of host processes (oracle/pool.py), about 10-20 s in all.
The reference's own workload is one 4096x4096 image (src/OCLTest.cpp:30,92-100), encoded stage
by stage as src/OCLEncoder.cpp:43-52 orders it."""
import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import pool as P
from roger_b200 import synth

pytestmark = pytest.mark.gpu
SEEDS = (100, 101, 102, 103)
REL_TOL_97 = 1e-4


@pytest.fixture(scope="module")
def C():
    from roger_b200 import codec
    return codec


@pytest.fixture(scope="module")
def oracle_streams():
    """Oracle codestreams of the two 4096x4096 images and of the 256 mixed images, encoded on
    every host core (spawned processes)."""
    mixed = synth.mixed_set(256)
    jobs = [("rgb", 4096, 4096, SEEDS, 6, 64, True), ("rgb", 4096, 4096, SEEDS, 6, 64, False)]
    jobs += [("mixed", d) for d in mixed]
    out = P.encode_many(jobs)
    return {"c1": out[0], "c2": out[1], "mixed": out[2:], "mixed_descs": mixed}


@pytest.fixture(scope="module")
def big_rgb():
    return synth.rgb(4096, 4096, SEEDS)


def test_c1_lossless_4096_codestream_equals_oracle(C, big_rgb, oracle_streams):
    enc = C.OCLEncoder(lossy=False)
    enc.run_rgb(torch.from_numpy(big_rgb).cuda(), levels=6, cbw=64, cbh=64)
    descs, data = enc.get_codeblocks()
    assert len(descs) == 12288
    cs = enc.codestream()
    ref = oracle_streams["c1"]
    assert len(cs) == len(ref)
    assert cs == ref, f"first difference at byte {next(i for i in range(len(ref)) if cs[i] != ref[i])}"
    back = C.decode_codestream(cs)
    assert np.array_equal(back.reshape(big_rgb.shape), big_rgb)


def test_c2_lossy_4096_indices_and_codestream_equal_oracle(C, big_rgb, oracle_streams):
    L = 6
    enc = C.OCLEncoder(lossy=True)
    enc.run_rgb(torch.from_numpy(big_rgb).cuda(), levels=L, cbw=64, cbh=64)
    q = enc.map_dwt_out()
    planes = O.planar_fwd(big_rgb, O.MCT_ICT, as_float=True)
    st = O.default_steps(4096, 4096, L)
    qref = np.stack([O.quantize(O.dwt97_fwd(p, L), L, st) for p in planes])
    assert np.array_equal(q, qref)
    cs = enc.codestream()
    assert cs == oracle_streams["c2"]
    # decode against the oracle's reconstruction (dequantise at the interval midpoint, inverse
    # 9/7, inverse ICT)
    rec = C.decode_codestream(cs).reshape(big_rgb.shape)
    ref = O.planar_inv(np.stack([O.dwt97_inv(O.dequantize(qq, L, st), L) for qq in qref]), O.MCT_ICT)
    assert np.array_equal(rec, ref.reshape(big_rgb.shape))


def test_c4_mixed_set_batched_codestreams_equal_oracle(oracle_streams):
    from roger_b200.batch import BatchEncoder
    descs = oracle_streams["mixed_descs"]
    imgs = [torch.from_numpy(synth.mixed_image(d)).cuda() for d in descs]
    be = BatchEncoder([dict(w=d["w"], h=d["h"], ncomp=d["ncomp"], kernel=d["kernel"], levels=d["levels"],
                            cb=d["cb"]) for d in descs])
    be.encode(imgs)
    bad = [i for i, d in enumerate(descs) if be.codestream(i) != oracle_streams["mixed"][i]]
    assert not bad, f"{len(bad)} of {len(descs)} images differ, first {descs[bad[0]]}"
    # the largest and the odd-sized images are in the set
    assert max(max(d["w"], d["h"]) for d in descs) >= 1500
    assert sum(1 for d in descs if d["w"] % 2 or d["h"] % 2) >= 64


def test_c4_mixed_set_batched_decode(C, oracle_streams):
    """The 256 codestreams decoded in one batched call (tier-2 on host threads, one tier-1
    launch over every block of every image): 5/3 images exactly the input, 9/7 images equal to
    the oracle's reconstruction (midpoint dequantisation, inverse 9/7, inverse ICT)."""
    descs = oracle_streams["mixed_descs"]
    outs = C.decode_codestreams(oracle_streams["mixed"])
    lossy = [d for d in descs if d["kernel"] == 97]
    recon = dict(zip((d["index"] for d in lossy), P.reconstruct_many(lossy)))
    bad = []
    for d, out in zip(descs, outs):
        ref = synth.mixed_image(d) if d["kernel"] == 53 else recon[d["index"]]
        if not np.array_equal(out.reshape(ref.shape), ref):
            bad.append(d)
    assert not bad, f"{len(bad)} of {len(descs)} images differ, first {bad[0]}"


@pytest.fixture(scope="module")
def c3_batch():
    return synth.float_batch(16, 1024, 1024, 200)


def test_c3_dwt97_16x1024_forward_inverse_bit_identical(C, c3_batch, capsys):
    L = 5
    x = torch.from_numpy(c3_batch).cuda()
    y = C.dwt_forward(x, L, 97, 0).cpu().numpy()
    back = C.dwt_inverse(torch.from_numpy(y).cuda(), L, 97, 0).cpu().numpy()
    worst = 0.0
    for i in range(16):
        ref = O.dwt97_fwd(c3_batch[i], L)
        assert np.array_equal(y[i], ref), f"image {i}: forward differs from the FP32 oracle"
        assert np.array_equal(back[i], O.dwt97_inv(ref, L)), f"image {i}: inverse differs from the FP32 oracle"
        if i < 2:
            r64 = O.dwt97_fwd(c3_batch[i].astype(np.float64), L, f64=True)
            for (x0, y0, sw, sh, o, lv) in O.subbands(1024, 1024, L):
                a, b = y[i, y0:y0 + sh, x0:x0 + sw], r64[y0:y0 + sh, x0:x0 + sw]
                worst = max(worst, float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-12)))
    with capsys.disabled():
        print(f"\nC3 9/7 FP32 vs FP64 (images 0-1, 16 subbands each): worst max|err|/max|coef| = {worst:.3e}")
    assert worst <= REL_TOL_97


def test_c3_rd_step_16x1024_matches_fp64_oracle(c3_batch):
    """One step of the config's rate-distortion loss on the whole batch (loss = MSE over every
    pixel + 0.01 * the rate of every image, image i's noise seeded with seed + i) against the
    FP64 oracle.

    The distortion term does not depend on the pixels (IDWT(DWT(x) + u*step) - x = IDWT(u*step)),
    so the pixel gradient is the rate term's alone, and log2(1 + |t|) has a kink at t = y/step +
    u = 0, where its gradient jumps by 2 * lam / (step * ln 2): for the few coefficients whose t
    lies within FP32 rounding of 0 the FP32 step and the FP64 oracle may take opposite sides of
    it (the config's finite-difference check uses a 64x64 crop for this reason).  So: the loss
    within 1e-5; the log-step gradients (sums over whole subbands) within 1e-4 relative; the
    pixel gradient within 1e-4 of its peak at all but a sliver of the pixels (below 1e-3 of
    them, each the image of such a kink)."""
    from roger_b200 import diff97 as D
    L, lam, seed, n = 5, 0.01, 200, 16
    ls = np.full(3 * L + 1, math.log(1 / 64.0))
    xt = torch.from_numpy(c3_batch).cuda().requires_grad_(True)
    lt = torch.from_numpy(ls.astype(np.float32)).cuda().requires_grad_(True)
    loss = D.rd_loss(xt, lt, L, lam, seed)
    loss.backward()
    gx = xt.grad.cpu().double().numpy()
    gl = lt.grad.cpu().double().numpy()
    # the oracle's loss is per image: loss_i = mse_i + lam * rate_i.  With lam = 0 it gives
    # mse_i alone, so the batch's loss sum_i (mse_i / n + lam * rate_i) follows, and so do its
    # gradients.
    tot, gl_ref, off = 0.0, np.zeros_like(ls), 0
    for i in range(n):
        xi = c3_batch[i].astype(np.float64)
        l1, g1, s1 = O.rd_loss(xi, L, ls, lam, seed + i)
        l0, g0, s0 = O.rd_loss(xi, L, ls, 0.0, seed + i)
        tot += l0 / n + (l1 - l0)
        gref = g0 / n + (g1 - g0)
        gl_ref += s0 / n + (s1 - s0)
        off += int((np.abs(gx[i] - gref) > 1e-4 * np.abs(gref).max()).sum())
    assert abs(loss.item() - tot) <= 1e-5 * abs(tot)
    assert np.abs(gl - gl_ref).max() <= 1e-4 * np.abs(gl_ref).max()
    assert off < 1e-3 * c3_batch.size, off
