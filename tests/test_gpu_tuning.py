"""GPU tests of the tuning surface: every MQ warp schedule gives the same codewords, and the
encoder's autotune keeps the result of the run it tuned on (rate-controlled runs included)."""
import numpy as np
import pytest

from roger_b200 import codec as C
from roger_b200 import synth
from roger_b200._lib import lib

pytestmark = pytest.mark.gpu


def _set_schedule(ctx, tiers, lanes):
    for k in range(4):
        w, l = tiers[k] if k < len(tiers) else (0, 0)
        assert lib().j2k_ctx_set_tuning(ctx.h, 6, (k << 24) | (l << 20) | w) == 0
    assert lib().j2k_ctx_set_tuning(ctx.h, 1, lanes) == 0


@pytest.mark.parametrize("tiers,lanes", [([], 8), ([], 32), ([(3, 1)], 16), ([(5, 1), (7, 3)], 8),
                                         ([(2, 1), (3, 2), (4, 5), (1, 8)], 32), ([(1000, 1)], 16)])
def test_every_mq_schedule_gives_the_same_codewords(tiers, lanes):
    img = synth.rgb(300, 260, (71, 72, 73, 74))
    ref = C.OCLEncoder(ctx=C.Context(0)).run_rgb(img, levels=4, cbw=32, cbh=32).get_codeblocks()
    ctx = C.Context(0)
    _set_schedule(ctx, tiers, lanes)
    for lossy in (False, True):
        enc = C.OCLEncoder(ctx=ctx, lossy=lossy)
        got = enc.run_rgb(img, levels=4, cbw=32, cbh=32).get_codeblocks()
        want = ref if not lossy else C.OCLEncoder(ctx=C.Context(0), lossy=True).run_rgb(
            img, levels=4, cbw=32, cbh=32).get_codeblocks()
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_encoder_autotune_keeps_the_result():
    img = synth.rgb(512, 384, (75, 76, 77, 78))
    enc = C.OCLEncoder(ctx=C.Context(0))
    cs = bytes(enc.run_rgb(img, levels=5).codestream())
    rep = enc.autotune(reps=1)
    assert rep["blocks_per_warp"] in (8, 16, 32)
    assert bytes(enc.codestream()) == cs
    assert bytes(enc.run_rgb(img, levels=5).codestream()) == cs
    cut = bytes(enc.run_rgb(img, levels=5, target_bytes=12000).codestream())
    assert len(cut) <= 12000
    enc.autotune(reps=1)
    assert bytes(enc.codestream()) == cut


@pytest.mark.parametrize("lanes", [2, 4, 8, 32])
def test_decoder_block_order_gives_the_same_image(lanes):
    """The tier-1 decoder's block-to-lane order (longest codewords first, J2K_TUNE_T1D_ORDER 1, or
    list order, 0) decodes every block the same: lossless round trips stay exact and the lossy
    decode is identical either way, unstyled and with the bypass / reset / per-pass styles."""
    img = synth.rgb(520, 300, (81, 82, 83, 84))
    for lossy, style in ((False, 0), (True, 0), (False, 7)):
        enc = C.OCLEncoder(ctx=C.Context(0), lossy=lossy)
        enc.run_rgb(img, levels=4, cbw=32, cbh=32, cblk_style=style)
        d, b = enc.get_codeblocks()
        pe = enc.get_pass_ends() if style else None
        outs = []
        for order in (0, 1):
            ctx = C.Context(0)
            assert lib().j2k_ctx_set_tuning(ctx.h, 10, lanes) == 0
            assert lib().j2k_ctx_set_tuning(ctx.h, 14, order) == 0
            dec = C.OCLDecoder(ctx=ctx, lossy=lossy)
            kw = {"cblk_style": style, "pass_ends": pe} if style else {}
            outs.append(np.array(dec.run(np.array(d), np.array(b), 520, 300, 3, levels=4, cbw=32, cbh=32, **kw)))
        assert np.array_equal(outs[0], outs[1])
        if not lossy:
            assert np.array_equal(outs[1], img)
