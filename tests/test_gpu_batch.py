"""GPU tests of the batched encoder: every image's codestream must be byte-identical to the
per-image encoder's (hence 9/7 PSNR identical) and to the CPU oracle's, with and without graph
replay and after autotuning."""
import io

import numpy as np
import pytest
import torch

from oracle import oracle as O
from roger_b200 import synth

pytestmark = pytest.mark.gpu


def _set(n=14, seed=7):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        w, h = int(rng.integers(33, 300)), int(rng.integers(33, 300))
        ncomp = 1 if i % 3 else 3
        kern = 53 if i % 2 == 0 else 97
        lv = int(min(max(int(np.floor(np.log2(min(w, h)))) - 3, 1), 5))
        cb = 32 if i % 4 < 2 else 64
        out.append(dict(w=w, h=h, ncomp=ncomp, kernel=kern, levels=lv, cb=cb, seed=1000 + i))
    return out


def _img(d):
    return synth.gray(d["w"], d["h"], d["seed"]) if d["ncomp"] == 1 else synth.rgb(d["w"], d["h"], (d["seed"],) * 4)


@pytest.fixture(scope="module")
def batch_and_images():
    from roger_b200.batch import BatchEncoder
    descs = _set()
    imgs = [_img(d) for d in descs]
    be = BatchEncoder(descs)
    be.encode(imgs)
    return be, descs, imgs


def test_batched_codestreams_match_per_image_and_oracle(batch_and_images):
    from roger_b200 import codec as C
    be, descs, imgs = batch_and_images
    for i, (d, img) in enumerate(zip(descs, imgs)):
        cs = be.codestream(i)
        enc = C.OCLEncoder(lossy=d["kernel"] == 97)
        enc.run_rgb(img, levels=d["levels"], cbw=d["cb"], cbh=d["cb"])
        assert cs == enc.codestream(), f"image {i} differs from the per-image path"
        assert cs == O.encode_image(img, d["levels"], d["cb"], d["cb"], d["kernel"] == 53), f"image {i} vs oracle"


def test_batched_lossless_decodes_exactly_in_openjpeg(batch_and_images):
    from PIL import Image
    be, descs, imgs = batch_and_images
    for i, (d, img) in enumerate(zip(descs, imgs)):
        if d["kernel"] != 53:
            continue
        dec = np.array(Image.open(io.BytesIO(be.codestream(i)))).reshape(img.shape)
        assert np.array_equal(dec, img)


def test_graph_replay_device_input_and_autotune_are_deterministic(batch_and_images):
    from roger_b200 import _lib
    be, descs, imgs = batch_and_images
    ref = [be.codestream(i) for i in range(len(descs))]
    be.encode(None)  # graph replay of the resident input
    assert [be.codestream(i) for i in range(len(descs))] == ref
    be.encode([torch.from_numpy(im).cuda() for im in imgs])  # device-side sources
    assert [be.codestream(i) for i in range(len(descs))] == ref
    be.set_option(_lib.J2K_BATCH_USE_GRAPH if hasattr(_lib, "J2K_BATCH_USE_GRAPH") else 1, 0)
    be.encode(None)
    assert [be.codestream(i) for i in range(len(descs))] == ref
    be.set_option(1, 1)
    rep = be.autotune(reps=1)
    assert set(rep) == {"tile53", "tile97", "phase_a_order", "mq", "phase_a_ctas_per_sm"}
    assert rep["phase_a_ctas_per_sm"] in (2, 3)
    be.encode(None)
    assert [be.codestream(i) for i in range(len(descs))] == ref


@pytest.mark.parametrize("tile", [0, 1, 2, 3])
def test_every_tile_shape_gives_identical_coefficients(batch_and_images, tile):
    be, descs, imgs = batch_and_images
    ref = [be.codestream(i) for i in range(len(descs))]
    be.set_option(2, tile)
    be.set_option(3, tile)
    be.encode(None)
    assert [be.codestream(i) for i in range(len(descs))] == ref


def test_bad_descriptor_is_rejected():
    from roger_b200.batch import BatchEncoder
    from roger_b200._lib import J2KError
    with pytest.raises(J2KError):
        BatchEncoder([dict(w=64, h=64, ncomp=2, kernel=53, levels=3, cb=64)])
    with pytest.raises(J2KError):
        BatchEncoder([dict(w=64, h=64, ncomp=1, kernel=53, levels=3, cb=48)])


def _same_blocks(got, be):
    assert len(got) == len(be.desc)
    for i, (d, b) in enumerate(got):
        rd, rb = be.codeblocks(i)
        assert np.array_equal(d, rd), f"image {i}: descriptors differ"
        assert np.array_equal(np.asarray(b), rb), f"image {i}: codeword bytes differ"


@pytest.mark.parametrize("pinned", [True, False])
def test_bulk_results_match_per_image_codeblocks(batch_and_images, pinned):
    be, descs, imgs = batch_and_images
    be.encode(imgs)
    _same_blocks(be.results(pinned=pinned), be)


def test_async_encode_is_read_by_the_pack(batch_and_images):
    be, descs, imgs = batch_and_images
    be.encode(imgs)
    ref = [(d.copy(), np.array(b)) for d, b in be.results()]
    be.encode(imgs, wait=False)
    got = be.results()
    for (d, b), (rd, rb) in zip(got, ref):
        assert np.array_equal(d, rd) and np.array_equal(np.asarray(b), rb)


@pytest.mark.parametrize("depth", [2, 3])
def test_streaming_encoder_matches_the_single_batch(batch_and_images, depth):
    from roger_b200.batch import StreamingBatchEncoder
    be, descs, imgs = batch_and_images
    be.encode(imgs)
    se = StreamingBatchEncoder(descs, depth=depth)
    pinned = StreamingBatchEncoder.pin(imgs)
    flipped = StreamingBatchEncoder.pin([np.ascontiguousarray(im[::-1]) for im in imgs])
    ref_flip = BatchEncoderRef(descs, flipped)
    seq = [pinned, flipped, pinned, pinned, flipped]
    n = 0
    for k, res in enumerate(se.run(seq)):
        want = be if seq[k] is pinned else ref_flip
        _same_blocks(res, want)
        n += 1
    assert n == len(seq)


def BatchEncoderRef(descs, imgs):
    from roger_b200.batch import BatchEncoder
    b = BatchEncoder(descs)
    b.encode(imgs)
    return b
