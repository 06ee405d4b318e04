"""CPU tests of the oracle itself: pinned by the golden fixtures and by an independent decoder
(OpenJPEG inside Pillow, run as a black box), plus round-trip properties."""
import hashlib
import io
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from roger_b200 import synth

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def _img(c):
    seed = tuple(c["seed"]) if isinstance(c["seed"], list) else c["seed"]
    return synth.gray(c["w"], c["h"], seed) if c["kind"] == "gray" else synth.rgb(c["w"], c["h"], seed)


def _decode(cs, shape):
    from PIL import Image
    return np.array(Image.open(io.BytesIO(cs))).reshape(shape)


@pytest.mark.parametrize("case", GOLD["codestreams"], ids=lambda c: c["name"])
def test_oracle_matches_golden_codestream(case):
    img = _img(case)
    assert hashlib.sha256(img.tobytes()).hexdigest() == case["image_sha256"], "generator drifted"
    cs = O.encode_image(img, case["levels"], case["cb"], case["cb"], case["lossless"])
    assert hashlib.sha256(cs).hexdigest() == case["codestream_sha256"]
    if "codestream_hex" in case:
        assert cs.hex() == case["codestream_hex"]


@pytest.mark.parametrize("case", [c for c in GOLD["codestreams"] if c["w"] * c["h"] <= 70000],
                         ids=lambda c: c["name"])
def test_openjpeg_decodes_oracle_codestream(case):
    img = _img(case)
    cs = O.encode_image(img, case["levels"], case["cb"], case["cb"], case["lossless"])
    dec = _decode(cs, img.shape)
    if case["lossless"]:
        assert np.array_equal(dec, img)
    else:
        d = dec.astype(float) - img
        psnr = 10 * np.log10(255.0 ** 2 / (d * d).mean())
        assert abs(psnr - case["openjpeg_psnr"]) < 1e-6


@pytest.mark.parametrize("w,h,nc,L,cb", [(1, 1, 1, 1, 64), (3, 5, 1, 1, 64), (65, 33, 1, 3, 32),
                                         (1, 50, 1, 2, 64), (50, 1, 3, 2, 32), (17, 91, 3, 4, 16),
                                         (128, 8, 1, 3, 4), (97, 97, 3, 5, 64)])
def test_openjpeg_lossless_edge_sizes(w, h, nc, L, cb):
    img = synth.gray(w, h, 7) if nc == 1 else synth.rgb(w, h, (1, 2, 3, 4))
    cs = O.encode_image(img, L, cb, cb, True)
    assert np.array_equal(_decode(cs, img.shape), img)


def test_ref_order_is_not_t800_invertible():
    """The reference's rows-first order gives different integer coefficients (so a T.800
    decoder does not invert it exactly), while the T.800 order round-trips in OpenJPEG."""
    img = synth.gray(96, 80, 3)
    cs_ref = O.encode_image(img, 3, 64, 64, True, O.ORDER_REF)
    assert not np.array_equal(_decode(cs_ref, img.shape), img)
    p = O.planar_fwd(img, O.MCT_NONE)[0]
    assert not np.array_equal(O.dwt53_fwd(p, 3, O.ORDER_REF), O.dwt53_fwd(p, 3, O.ORDER_T800))


@pytest.mark.parametrize("order", [O.ORDER_T800, O.ORDER_REF])
@pytest.mark.parametrize("w,h,L", [(1, 1, 1), (2, 3, 2), (64, 64, 6), (129, 67, 5), (31, 200, 4)])
def test_dwt53_round_trip(order, w, h, L):
    x = (np.random.default_rng(w * h).integers(-300, 300, (h, w))).astype(np.int32)
    c = O.dwt53_fwd(x, L, order)
    assert np.array_equal(O.dwt53_inv(c, L, order), x)


@pytest.mark.parametrize("w,h,L", [(1, 1, 1), (2, 3, 2), (64, 64, 5), (129, 67, 5)])
def test_dwt97_round_trip_and_fp64_agreement(w, h, L):
    x = np.random.default_rng(5).uniform(-128, 128, (h, w))
    c32 = O.dwt97_fwd(x.astype(np.float32), L)
    c64 = O.dwt97_fwd(x, L, f64=True)
    rel = np.abs(c32 - c64).max() / max(np.abs(c64).max(), 1e-30)
    assert rel < 1e-5
    back = O.dwt97_inv(c64, L, f64=True)
    assert np.abs(back - x).max() < 1e-9


def test_dwt97_adjoint_is_exact_transpose():
    w, h, L = 13, 11, 3
    n = w * h
    F = np.zeros((n, n))
    I = np.zeros((n, n))
    Fa = np.zeros((n, n))
    Ia = np.zeros((n, n))
    for i in range(n):
        e = np.zeros(n)
        e[i] = 1.0
        F[:, i] = O.dwt97_fwd(e.reshape(h, w), L, f64=True).ravel()
        I[:, i] = O.dwt97_inv(e.reshape(h, w), L, f64=True).ravel()
        Fa[:, i] = O.dwt97_fwd_adj(e.reshape(h, w), L).ravel()
        Ia[:, i] = O.dwt97_inv_adj(e.reshape(h, w), L).ravel()
    assert np.abs(Fa - F.T).max() < 1e-12
    assert np.abs(Ia - I.T).max() < 1e-12
    assert np.abs(I @ F - np.eye(n)).max() < 1e-9


def test_rd_loss_gradient_matches_fd64():
    x = synth.gray(24, 20, 11).astype(np.float64) / 255.0
    L = 3
    ls = np.full(3 * L + 1, np.log(1 / 64.0))
    loss, gx, gl = O.rd_loss(x, L, ls, 0.01, 1234)
    h = 1e-6
    rng = np.random.default_rng(0)
    for _ in range(6):
        i, j = rng.integers(0, 20), rng.integers(0, 24)
        xp, xm = x.copy(), x.copy()
        xp[i, j] += h
        xm[i, j] -= h
        fd = (O.rd_loss(xp, L, ls, 0.01, 1234, False) - O.rd_loss(xm, L, ls, 0.01, 1234, False)) / (2 * h)
        assert abs(fd - gx[i, j]) <= 1e-4 * max(abs(fd), 1e-3)
    for b in range(len(ls)):
        lp, lm = ls.copy(), ls.copy()
        lp[b] += h
        lm[b] -= h
        fd = (O.rd_loss(x, L, lp, 0.01, 1234, False) - O.rd_loss(x, L, lm, 0.01, 1234, False)) / (2 * h)
        assert abs(fd - gl[b]) <= 1e-4 * max(abs(fd), 1e-3)


@pytest.mark.parametrize("t", GOLD["t1"], ids=lambda t: t["tag"])
def test_t1_golden_vectors_and_round_trip(t):
    blk = np.array(t["coeff"], np.int32).reshape(t["ch"], t["cw"])
    data, info, syms = O.t1_encode(blk, t["orient"], want_symbols=True)
    assert data.hex() == t["codeword_hex"]
    assert info["numbps"] == t["numbps"] and info["nsyms"] == t["nsyms"]
    assert hashlib.sha256(syms.tobytes()).hexdigest() == t["symbols_sha256"]
    back = O.t1_decode(data, info["numbps"], info["npasses"], t["orient"], t["cw"], t["ch"])
    assert np.array_equal(back, blk)


@pytest.mark.parametrize("orient", [0, 1, 2, 3])
@pytest.mark.parametrize("cw,ch", [(64, 64), (32, 32), (5, 7), (64, 3), (1, 1), (4, 64)])
def test_t1_round_trip_random(orient, cw, ch):
    rng = np.random.default_rng(cw * 100 + ch + orient)
    blk = (rng.laplace(0, 20, (ch, cw))).astype(np.int32)
    blk[rng.random((ch, cw)) < 0.3] = 0
    data, info = O.t1_encode(blk, orient)
    assert np.array_equal(O.t1_decode(data, info["numbps"], info["npasses"], orient, cw, ch), blk)


def test_quantiser_round_trip():
    L = 3
    c = np.random.default_rng(1).normal(0, 30, (40, 36)).astype(np.float32)
    st = O.default_steps(36, 40, L)
    q = O.quantize(c, L, st)
    r = O.dequantize(q, L, st)
    for (x0, y0, sw, sh, o, lv), s in zip(O.subbands(36, 40, L), st):
        blk = c[y0:y0 + sh, x0:x0 + sw]
        assert np.all(np.abs(r[y0:y0 + sh, x0:x0 + sw] - blk) <= s + 1e-6)


def test_rct_ict_round_trip():
    img = synth.rgb(37, 21, (1, 2, 3, 4))
    assert np.array_equal(O.planar_inv(O.planar_fwd(img, O.MCT_RCT), O.MCT_RCT), img)
    back = O.planar_inv(O.planar_fwd(img, O.MCT_ICT, as_float=True), O.MCT_ICT)
    assert np.abs(back.astype(int) - img).max() <= 1


def test_philox_known_answers_and_noise_layout():
    """Philox4x32-10 against the published known-answer vectors of its authors (Random123), and
    the relaxed quantiser's layout: one block per 4 samples of a row, word x % 4."""
    import ctypes as C
    L = O.lib()
    L.or_philox4x32.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    kat = [((0, 0), (0, 0, 0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
           ((0xffffffff, 0xffffffff), (0xffffffff,) * 4, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
           ((0xa4093822, 0x299f31d0), (0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344),
            (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for key, ctr, want in kat:
        c, o = (C.c_uint32 * 4)(*ctr), (C.c_uint32 * 4)()
        L.or_philox4x32(key[0], key[1], c, o)
        assert tuple(o) == want
    seed, w = 12345, 10
    for x, y in [(0, 0), (3, 0), (4, 0), (9, 2), (7, 5)]:
        ctr = y * ((w + 3) // 4) + x // 4
        c, o = (C.c_uint32 * 4)(ctr & 0xffffffff, ctr >> 32, 0, 0), (C.c_uint32 * 4)()
        L.or_philox4x32(seed & 0xffffffff, seed >> 32, c, o)
        assert O.rd_noise(seed, w, x, y) == (o[x % 4] >> 8) / 16777216.0 - 0.5


STYLES = [0, O.STYLE_BYPASS, O.STYLE_RESET, O.STYLE_TERMALL, O.STYLE_RESET | O.STYLE_TERMALL,
          O.STYLE_BYPASS | O.STYLE_TERMALL, O.STYLE_BYPASS | O.STYLE_RESET,
          O.STYLE_BYPASS | O.STYLE_RESET | O.STYLE_TERMALL]


def test_style_pass_rules():
    """Raw passes: SPP and MRP from the fifth bit-plane on (pass 10 on) under bypass; the
    codeword ends after every pass under termination, else where bypass switches between raw
    and MQ coding, and always after the last pass (T.800 D.6, Table A.19)."""
    assert [p for p in range(20) if O.pass_raw(O.STYLE_BYPASS, p)] == [10, 11, 13, 14, 16, 17, 19]
    assert not any(O.pass_raw(O.STYLE_RESET | O.STYLE_TERMALL, p) for p in range(40))
    assert [p for p in range(16) if O.pass_terminated(O.STYLE_BYPASS, p, 16)] == [9, 11, 12, 14, 15]
    assert [p for p in range(16) if O.pass_terminated(0, p, 16)] == [15]
    assert all(O.pass_terminated(O.STYLE_TERMALL, p, 16) for p in range(16))


@pytest.mark.parametrize("style", STYLES)
def test_styled_blocks_round_trip(style):
    """Every style: the styled encoder's codeword decodes back to the block (segments located
    by the pass ends), and style 0 gives the plain encoder's codeword."""
    rng = np.random.default_rng(style + 11)
    for cw, ch, orient in [(64, 64, 0), (32, 32, 3), (17, 5, 1), (4, 4, 2), (1, 1, 0), (64, 3, 1), (8, 64, 2)]:
        blk = rng.integers(-5000, 5000, (ch, cw)).astype(np.int32)
        blk[rng.random((ch, cw)) < 0.6] = 0
        data, info, pe = O.t1_encode_styled(blk, orient, style)
        assert pe[-1] == len(data) if info["npasses"] else len(data) == 0
        back = O.t1_decode_styled(data, pe, info["numbps"], info["npasses"], orient, cw, ch, style)
        assert np.array_equal(back, blk), (cw, ch)
        if style == 0:
            assert data == O.t1_encode(blk, orient)[0]


@pytest.mark.parametrize("style", STYLES[1:])
def test_openjpeg_decodes_styled_oracle_codestreams(style):
    """An independent decoder (OpenJPEG through Pillow) decodes the styled codestreams: lossless
    exactly, lossy to the same pixels as the unstyled stream."""
    from PIL import Image
    for w, h, nc, lossless, L, cb in [(200, 131, 3, True, 4, 32), (256, 256, 3, False, 5, 64),
                                      (67, 45, 1, False, 3, 16), (97, 200, 1, True, 5, 64)]:
        img = synth.gray(w, h, 3) if nc == 1 else synth.rgb(w, h, (5, 6, 7, 8))
        cs = O.encode_image(img, L, cb, cb, lossless, style=style)
        dec = np.array(Image.open(io.BytesIO(cs))).reshape(img.shape)
        ref = np.array(Image.open(io.BytesIO(O.encode_image(img, L, cb, cb, lossless)))).reshape(img.shape)
        assert np.array_equal(dec, ref)
        if lossless:
            assert np.array_equal(dec, img)
        assert cs[cs.index(b"\xff\x52") + 12] == style  # COD code-block style byte
