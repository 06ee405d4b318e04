"""Tier-2 reading: codestreams written by this library (the oracle's, byte-identical to the GPU
encoder's) and by OpenJPEG (through Pillow, a black box) are parsed by j2k_codestream_read;
the code-blocks are then decoded (tier-1, inverse DWT, inverse colour transform) by the oracle
on the CPU here and by the GPU decoder in the -m gpu test, and must give the input back exactly
(lossless) or what OpenJPEG itself decodes to within rounding (lossy)."""
import io

import numpy as np
import pytest
import torch

from oracle import oracle as O
from roger_b200 import codec as C
from roger_b200 import synth
from roger_b200._lib import J2KError

PIL = pytest.importorskip("PIL.Image")


def _openjpeg(img, levels, lossless=True, cb=64):
    buf = io.BytesIO()
    kw = dict(irreversible=not lossless, num_resolutions=levels + 1, codeblock_size=(cb, cb), progression="LRCP",
              no_jp2=True)
    if img.ndim == 3:
        kw["mct"] = 1
    PIL.fromarray(img).save(buf, "JPEG2000", **kw)
    return buf.getvalue()


def _cpu_decode(cs):
    info, descs, data = C.read_codestream(cs)
    w, h, nc, L = info["w"], info["h"], info["ncomp"], info["levels"]
    planes = np.zeros((nc, h, w), np.int32)
    for d in descs:
        if d["length"] <= 0 and d["npasses"] == 0:
            continue
        blk = O.t1_decode(bytes(data[d["offset"]:d["offset"] + d["length"]]), int(d["numbps"]), int(d["npasses"]),
                          int(d["orient"]), int(d["cw"]), int(d["ch"]))
        planes[d["comp"], d["y0"]:d["y0"] + d["ch"], d["x0"]:d["x0"] + d["cw"]] = blk
    if info["lossless"]:
        rec = np.stack([O.dwt53_inv(p, L) for p in planes])
        return O.planar_inv(rec, 1 if nc == 3 else 0).reshape(h, w, nc) if nc == 3 else \
            O.planar_inv(rec, 0).reshape(h, w)
    st = info["steps"]
    rec = np.stack([O.dwt97_inv(O.dequantize(p, L, st), L) for p in planes])
    out = O.planar_inv(rec, 2 if nc == 3 else 0)
    return out.reshape(h, w, nc) if nc == 3 else out.reshape(h, w)


CASES = [(131, 97, 1, 4, 64), (200, 64, 3, 5, 64), (77, 301, 3, 3, 32), (64, 64, 1, 2, 32)]


@pytest.mark.parametrize("w,h,nc,L,cb", CASES)
def test_own_codestream_parses_and_round_trips(w, h, nc, L, cb):
    img = synth.gray(w, h, 5) if nc == 1 else synth.rgb(w, h, (5, 6, 7, 8))
    cs = bytes(O.encode_image(img, L, cb, cb, True))
    info, descs, data = C.read_codestream(cs)
    assert (info["w"], info["h"], info["ncomp"], info["levels"], info["cbw"]) == (w, h, nc, L, cb)
    assert info["lossless"] and info["mct"] == (1 if nc == 3 else 0)
    assert np.array_equal(_cpu_decode(cs).reshape(img.shape), img)


@pytest.mark.parametrize("w,h,nc,L,cb", CASES)
def test_openjpeg_lossless_codestream_decodes_exactly(w, h, nc, L, cb):
    img = synth.gray(w, h, 9) if nc == 1 else synth.rgb(w, h, (9, 10, 11, 12))
    cs = _openjpeg(img, L, True, cb)
    assert np.array_equal(_cpu_decode(cs).reshape(img.shape), img)


def test_openjpeg_lossy_codestream_matches_openjpeg_decode():
    img = synth.rgb(160, 120, (21, 22, 23, 24))
    cs = _openjpeg(img, 4, lossless=False)
    ours = _cpu_decode(cs).reshape(img.shape).astype(np.int32)
    theirs = np.asarray(PIL.open(io.BytesIO(cs))).astype(np.int32)
    assert np.abs(ours - theirs).max() <= 2


def test_unsupported_streams_are_rejected_with_a_reason():
    img = synth.rgb(64, 64, (1, 2, 3, 4))
    buf = io.BytesIO()
    PIL.fromarray(img).save(buf, "JPEG2000", num_resolutions=3, tile_size=(32, 32), irreversible=False, mct=1,
                            no_jp2=True)
    with pytest.raises(J2KError, match="tile"):
        C.read_codestream(buf.getvalue())
    buf = io.BytesIO()
    PIL.fromarray(img).save(buf, "JPEG2000", num_resolutions=3, irreversible=False, mct=0, no_jp2=True)
    with pytest.raises(J2KError, match="colour transform"):
        C.read_codestream(buf.getvalue())
    with pytest.raises(J2KError):
        C.read_codestream(b"\x00\x01\x02")


def test_sizes_beyond_16_bits_are_refused():
    """Code-block positions are kept in 16 bits (the writer's limit too), so a SIZ width or
    height above 65535, or of 0, is refused instead of decoding to wrapped positions."""
    cs = bytearray(O.encode_image(synth.gray(64, 48, 0), 2, 32, 32, True))
    siz = cs.index(b"\xff\x51")
    for w, h in [(70000, 48), (64, 65536), (0, 48), (1 << 31, 1 << 31)]:
        bad = bytearray(cs)
        bad[siz + 6:siz + 10] = w.to_bytes(4, "big")    # Xsiz
        bad[siz + 10:siz + 14] = h.to_bytes(4, "big")   # Ysiz
        bad[siz + 22:siz + 26] = w.to_bytes(4, "big")   # XTsiz (one tile)
        bad[siz + 26:siz + 30] = h.to_bytes(4, "big")   # YTsiz
        with pytest.raises(J2KError, match="65535"):
            C.read_codestream(bytes(bad))


def _openjpeg_layers(img, levels, rates, prog="LRCP", cb=64):
    buf = io.BytesIO()
    kw = dict(irreversible=False, num_resolutions=levels + 1, codeblock_size=(cb, cb), progression=prog,
              quality_mode="rates", quality_layers=rates, no_jp2=True)
    if img.ndim == 3:
        kw["mct"] = 1
    PIL.fromarray(img).save(buf, "JPEG2000", **kw)
    return buf.getvalue()


@pytest.mark.parametrize("prog", ["LRCP", "RLCP"])
@pytest.mark.parametrize("w,h,nc,L,cb", CASES[:3])
def test_openjpeg_multilayer_lossless_decodes_exactly(w, h, nc, L, cb, prog):
    img = synth.gray(w, h, 41) if nc == 1 else synth.rgb(w, h, (41, 42, 43, 44))
    cs = _openjpeg_layers(img, L, [30, 8, 0], prog, cb)
    info, descs, data = C.read_codestream(cs)
    assert info["layers"] == 3
    assert np.array_equal(_cpu_decode(cs).reshape(img.shape), img)
    # the first layers give each block a prefix of its full codeword and fewer passes
    prev = None
    for keep in (1, 2, 3):
        _, d, b = C.read_codestream(cs, max_layers=keep)
        assert np.all(d["npasses"] <= descs["npasses"]) and np.all(d["length"] <= descs["length"])
        for k in np.flatnonzero(d["length"] > 0)[:200]:
            full = data[descs["offset"][k]:descs["offset"][k] + d["length"][k]]
            assert np.array_equal(b[d["offset"][k]:d["offset"][k] + d["length"][k]], full)
        if prev is not None:
            assert np.all(d["npasses"] >= prev)
        prev = d["npasses"].copy()
    assert np.array_equal(prev, descs["npasses"])


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,nc,L,cb", CASES)
def test_gpu_decodes_openjpeg_and_own_codestreams(w, h, nc, L, cb):
    img = synth.gray(w, h, 13) if nc == 1 else synth.rgb(w, h, (13, 14, 15, 16))
    for cs in (_openjpeg(img, L, True, cb), bytes(O.encode_image(img, L, cb, cb, True))):
        out = C.decode_codestream(cs)
        assert np.array_equal(out.reshape(img.shape), img)


@pytest.mark.gpu
def test_batched_decode_matches_per_image():
    streams = []
    for w, h, nc, L, cb in CASES:
        img = synth.gray(w, h, 61) if nc == 1 else synth.rgb(w, h, (61, 62, 63, 64))
        streams += [_openjpeg(img, L, True, cb), bytes(O.encode_image(img, L, cb, cb, True)),
                    _openjpeg_layers(img, L, [30, 8, 0], "RLCP", cb)]
    img = synth.rgb(160, 120, (65, 66, 67, 68))
    streams.append(_openjpeg(img, 4, lossless=False))
    enc = C.OCLEncoder(lossy=True)
    streams.append(bytes(enc.run_rgb(img, levels=4).codestream()))
    enc = C.OCLEncoder(lossy=False)
    streams.append(bytes(enc.run_rgb(img, levels=4, cbw=32, cbh=32, target_bytes=4000).codestream()))
    outs = C.decode_codestreams(streams)
    assert len(outs) == len(streams)
    for k, (cs, out) in enumerate(zip(streams, outs)):
        ref = C.decode_codestream(cs)
        assert np.array_equal(out.reshape(-1), ref.reshape(-1)), f"stream {k}"
    # only the first layer of the layered streams
    first = C.decode_codestreams(streams[2:3], max_layers=1)[0]
    assert np.array_equal(first.reshape(-1), C.decode_codestream(streams[2], max_layers=1).reshape(-1))


@pytest.mark.parametrize("w,h,nc,L,cb", CASES)
def test_header_info_matches_the_full_parse(w, h, nc, L, cb):
    img = synth.gray(w, h, 31) if nc == 1 else synth.rgb(w, h, (31, 32, 33, 34))
    for cs in (_openjpeg(img, L, True, cb), bytes(O.encode_image(img, L, cb, cb, True)),
               _openjpeg_layers(img, L, [30, 8, 0], "RLCP", cb)):
        head = C.codestream_info(cs)
        full = C.read_codestream(cs)[0]
        assert all(head[k] == full[k] for k in head)


@pytest.mark.parametrize("style", [1, 2, 4, 5, 6, 7])
@pytest.mark.parametrize("w,h,nc,L,cb,lossless", [(200, 131, 3, 4, 32, True), (97, 64, 1, 5, 16, True),
                                                  (128, 96, 3, 3, 64, False)])
def test_styled_oracle_codestreams_parse_and_decode(style, w, h, nc, L, cb, lossless):
    """Streams in the bypass / reset / per-pass termination styles: the reader gives the
    style and each block's pass ends, and the oracle's styled block decoder, fed those segments,
    rebuilds the coefficients, hence the image (lossless) or OpenJPEG's decode (lossy)."""
    img = synth.gray(w, h, 3) if nc == 1 else synth.rgb(w, h, (5, 6, 7, 8))
    cs = O.encode_image(img, L, cb, cb, lossless, style=style)
    info, descs, data = C.read_codestream(cs)
    assert info["cblk_style"] == style
    pe = C.read_pass_ends(cs)
    assert pe.shape == (len(descs), 92)
    planes = np.zeros((nc, h, w), np.int32)
    for d, ends in zip(descs, pe):
        if d["npasses"] == 0:
            continue
        seg = bytes(data[d["offset"]:d["offset"] + d["length"]])
        assert ends[d["npasses"] - 1] == d["length"]
        blk = O.t1_decode_styled(seg, ends[:d["npasses"]], int(d["numbps"]), int(d["npasses"]), int(d["orient"]),
                                 int(d["cw"]), int(d["ch"]), style)
        planes[d["comp"], d["y0"]:d["y0"] + d["ch"], d["x0"]:d["x0"] + d["cw"]] = blk
    if lossless:
        rec = np.stack([O.dwt53_inv(p, L) for p in planes])
        out = O.planar_inv(rec, 1 if nc == 3 else 0)
        assert np.array_equal(out.reshape(img.shape), img)
    else:
        st = info["steps"]
        rec = np.stack([O.dwt97_inv(O.dequantize(p, L, st), L) for p in planes])
        out = O.planar_inv(rec, 2).reshape(img.shape)
        ref = np.array(PIL.open(io.BytesIO(cs))).reshape(img.shape)
        assert np.abs(out.astype(int) - ref.astype(int)).max() <= 1


def test_unsupported_code_block_styles_are_refused():
    cs = bytearray(O.encode_image(synth.gray(64, 48, 0), 2, 32, 32, True))
    cod = cs.index(b"\xff\x52")
    for sty, word in [(0x08, "causal"), (0x20, "segmentation")]:
        bad = bytearray(cs)
        bad[cod + 12] = sty
        with pytest.raises(J2KError, match=word):
            C.read_codestream(bytes(bad))
