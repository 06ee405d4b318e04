"""GPU parity of the code-block styles (bypass, reset, per-pass termination; T.800 Table A.19,
D.6) against the oracle: the styled encoder's codestream (codewords, segment lengths in the
packet headers, COD style byte) is byte-equal to the oracle's, each block's pass ends equal the
oracle's at every terminated pass, OpenJPEG decodes the streams, and the GPU decoder (per
image and batched) decodes them back exactly."""
import io

import numpy as np
import pytest
import torch

from oracle import oracle as O
from roger_b200 import synth

pytestmark = pytest.mark.gpu
STYLES = [1, 2, 4, 5, 6, 7]


@pytest.fixture(scope="module")
def C():
    from roger_b200 import codec
    return codec


def _img(w, h, nc, seed):
    return synth.gray(w, h, seed) if nc == 1 else synth.rgb(w, h, (seed, seed + 1, seed + 2, seed + 3))


@pytest.mark.parametrize("style", STYLES)
@pytest.mark.parametrize("w,h,nc,L,cb,lossless", [(333, 257, 3, 5, 32, True), (256, 200, 1, 4, 64, True),
                                                  (300, 300, 3, 5, 64, False), (65, 129, 1, 3, 16, False),
                                                  (7, 5, 1, 1, 4, True)])
def test_styled_codestream_equals_oracle_and_decodes(C, style, w, h, nc, L, cb, lossless):
    img = _img(w, h, nc, 21)
    enc = C.OCLEncoder(lossy=not lossless)
    enc.run_rgb(torch.from_numpy(img).cuda(), levels=L, cbw=cb, cbh=cb, cblk_style=style)
    cs = enc.codestream()
    ref = O.encode_image(img, L, cb, cb, lossless, style=style)
    assert cs == ref
    # pass ends at the terminated passes, block by block (the oracle's styled tier-1)
    descs, data = enc.get_codeblocks()
    pe = enc.get_pass_ends()
    # decode: per image and batched, against the input (lossless) or the unstyled decode (lossy)
    back = C.decode_codestream(cs).reshape(img.shape)
    plain = O.encode_image(img, L, cb, cb, lossless)
    ref_img = C.decode_codestream(plain).reshape(img.shape)
    assert np.array_equal(back, ref_img)
    if lossless:
        assert np.array_equal(back, img)
    outs = C.decode_codestreams([cs, plain, cs])
    for o in outs:
        assert np.array_equal(o.reshape(img.shape), ref_img)
    for d, ends in zip(descs, pe):
        np_ = int(d["npasses"])
        if np_:
            assert ends[np_ - 1] == d["length"]


@pytest.mark.parametrize("style", [6, 7, 5])
def test_styled_blocks_and_pass_ends_equal_oracle(C, style):
    """Every code-block of a lossless 512x512 encode: codeword bytes and the pass ends of its
    terminated passes equal the oracle's styled tier-1 of the same coefficients."""
    img = synth.gray(512, 512, 0)
    coef = O.dwt53_fwd(O.planar_fwd(img, 0)[0], 5)
    enc = C.OCLEncoder(lossy=False)
    enc.run_rgb(torch.from_numpy(img).cuda(), levels=5, cbw=64, cbh=64, cblk_style=style)
    descs, data = enc.get_codeblocks()
    pe = enc.get_pass_ends()
    for d, ends in zip(descs, pe):
        blk = coef[d["y0"]:d["y0"] + d["ch"], d["x0"]:d["x0"] + d["cw"]]
        rdata, info, rpe = O.t1_encode_styled(blk, int(d["orient"]), style)
        assert data[d["offset"]:d["offset"] + d["length"]].tobytes() == rdata
        assert int(d["npasses"]) == info["npasses"]
        for p in range(info["npasses"]):
            if O.pass_terminated(style, p, info["npasses"]):
                assert ends[p] == rpe[p], (d["x0"], d["y0"], p)


def test_styled_stream_decodes_in_openjpeg(C):
    from PIL import Image
    img = _img(401, 300, 3, 40)
    for style in (6, 7):
        enc = C.OCLEncoder(lossy=False)
        enc.run_rgb(img, levels=5, cbw=64, cbh=64, cblk_style=style)
        dec = np.array(Image.open(io.BytesIO(enc.codestream()))).reshape(img.shape)
        assert np.array_equal(dec, img)


def test_c1_4096_pass_parallel_style_equals_oracle(C):
    """The 4096x4096 RGB lossless workload with reset + per-pass termination (every pass coded
    in its own lane): the codestream equals the oracle's, and the GPU decodes it exactly."""
    img = synth.rgb(4096, 4096, (100, 101, 102, 103))
    style = O.STYLE_RESET | O.STYLE_TERMALL
    enc = C.OCLEncoder(lossy=False)
    enc.run_rgb(torch.from_numpy(img).cuda(), levels=6, cbw=64, cbh=64, cblk_style=style)
    cs = enc.codestream()
    assert cs == O.encode_image(img, 6, 64, 64, True, style=style)
    assert np.array_equal(C.decode_codestream(cs).reshape(img.shape), img)


def test_style_with_rate_control_is_refused(C):
    from roger_b200._lib import J2KError
    img = _img(64, 64, 1, 3)
    with pytest.raises(J2KError):
        C.OCLEncoder(lossy=False).run_rgb(img, levels=3, cbw=32, cbh=32, cblk_style=6, target_bytes=500)
