"""Host tier-2 writer (j2k_codestream_write), on the CPU: code-blocks coded by the oracle's
tier-1 are written into codestreams.  One layer must be byte-identical to the oracle's own
codestream; quality layers (cut at the oracle's bit-plane truncation points) must parse back
through j2k_codestream_read_layers to exactly the passes and bytes written, decode losslessly
in OpenJPEG when complete, and decode each prefix of layers like the oracle's decode of the same
cuts (OpenJPEG: within 1 dB)."""
import io

import numpy as np
import pytest

from oracle import oracle as O
from roger_b200 import _lib as L
from roger_b200 import codec as C
from roger_b200 import synth
from roger_b200._lib import J2KError

PIL = pytest.importorskip("PIL.Image")


def _blocks(img, levels, cb):
    """Oracle tier-1 of every code-block of the lossless transform, in job order."""
    h, w = img.shape[:2]
    nc = 1 if img.ndim == 2 else img.shape[2]
    planes = O.planar_fwd(img, 1 if nc == 3 else 0)
    descs, datas, infos, coefs = [], [], [], []
    off = 0
    for c in range(nc):
        co = O.dwt53_fwd(planes[c], levels)
        coefs.append(co)
        for b, (x0, y0, sw, sh, o, lv) in enumerate(O.subbands(w, h, levels)):
            if not sw or not sh:
                continue
            for by in range(0, sh, cb):
                for bx in range(0, sw, cb):
                    blk = co[y0 + by:y0 + min(by + cb, sh), x0 + bx:x0 + min(bx + cb, sw)]
                    data, info = O.t1_encode(blk, o)
                    d = np.zeros(1, L.CB_DESC)[0]
                    d["offset"], d["length"], d["numbps"], d["npasses"] = off, info["length"], info["numbps"], info["npasses"]
                    d["orient"], d["band"], d["x0"], d["y0"] = o, b, x0 + bx, y0 + by
                    d["cw"], d["ch"], d["comp"] = blk.shape[1], blk.shape[0], c
                    descs.append(d)
                    datas.append(data)
                    infos.append(info)
                    off += len(data)
    return np.array(descs, L.CB_DESC), np.frombuffer(b"".join(datas), np.uint8), infos, coefs


# the last two have 4096 code-blocks or more, so the writer builds each layer's packets on host
# threads
CASES = [(96, 80, 3, 3, 32), (131, 97, 1, 4, 64), (200, 64, 3, 5, 64), (512, 512, 1, 5, 8),
         (384, 384, 3, 4, 8)]


@pytest.mark.parametrize("w,h,nc,lv,cb", CASES)
def test_one_layer_is_the_oracles_codestream(w, h, nc, lv, cb):
    img = synth.gray(w, h, 91) if nc == 1 else synth.rgb(w, h, (91, 92, 93, 94))
    descs, data, _, _ = _blocks(img, lv, cb)
    cs = C.write_codestream(w, h, nc, lv, descs, data, cb, cb)
    assert cs == bytes(O.encode_image(img, lv, cb, cb, True))


def _layers(descs, infos, cuts):
    """(L, n) passes and lengths: layer l cuts block i after bit-plane cuts[l](numbps) (None: all)."""
    n = len(descs)
    npl = np.zeros((len(cuts), n), np.int32)
    lnl = np.zeros((len(cuts), n), np.int32)
    for i, info in enumerate(infos):
        nb = info["numbps"]
        for l, cut in enumerate(cuts):
            if nb == 0:
                continue
            k = nb - 1 if cut is None else min(cut(nb), nb - 1)
            if k < 0:
                continue
            npl[l, i] = min(3 * k + 1, info["npasses"])
            lnl[l, i] = O.truncation_length(info, k)
    return npl, lnl


def _oracle_decode(img_shape, lv, descs, data):
    h, w = img_shape[:2]
    nc = 1 if len(img_shape) == 2 else img_shape[2]
    planes = np.zeros((nc, h, w), np.int32)
    for d in descs:
        if d["npasses"] == 0:
            continue
        blk = O.t1_decode(bytes(data[d["offset"]:d["offset"] + d["length"]]), int(d["numbps"]), int(d["npasses"]),
                          int(d["orient"]), int(d["cw"]), int(d["ch"]))
        planes[d["comp"], d["y0"]:d["y0"] + d["ch"], d["x0"]:d["x0"] + d["cw"]] = blk
    rec = np.stack([O.dwt53_inv(p, lv) for p in planes])
    return O.planar_inv(rec, 1 if nc == 3 else 0).reshape(img_shape)


def _psnr(a, b):
    e = a.astype(np.float64) - b.astype(np.float64)
    return 10 * np.log10(255.0 ** 2 / max((e * e).mean(), 1e-12))


@pytest.mark.parametrize("w,h,nc,lv,cb", CASES)
def test_quality_layers_round_trip(w, h, nc, lv, cb):
    img = synth.gray(w, h, 95) if nc == 1 else synth.rgb(w, h, (95, 96, 97, 98))
    descs, data, infos, _ = _blocks(img, lv, cb)
    cuts = [lambda nb: 0, lambda nb: nb // 2, None]
    npl, lnl = _layers(descs, infos, cuts)
    cs = C.write_codestream(w, h, nc, lv, descs, data, cb, cb, layers=(npl, lnl))
    info, full, fdata = C.read_codestream(cs)
    assert info["layers"] == 3
    # complete stream: lossless, ours and OpenJPEG's
    assert np.array_equal(_oracle_decode(img.shape, lv, full, fdata), img)
    assert np.array_equal(np.asarray(PIL.open(io.BytesIO(cs))).reshape(img.shape), img)
    last = -1.0
    for keep in (1, 2):
        _, d, b = C.read_codestream(cs, max_layers=keep)
        assert np.array_equal(d["npasses"], npl[keep - 1]) and np.array_equal(d["length"], lnl[keep - 1])
        for k in range(len(d)):
            n = int(d["length"][k])
            assert bytes(b[d["offset"][k]:d["offset"][k] + n]) == bytes(data[descs["offset"][k]:descs["offset"][k] + n])
        ours = _oracle_decode(img.shape, lv, d, b)
        p = _psnr(ours, img)
        assert p > last
        last = p
        im = PIL.open(io.BytesIO(cs))
        t = im.tile[0]
        im.tile = [type(t)(t[0], t[1], t[2], (t[3][0], 0, keep) + tuple(t[3][3:]))]
        theirs = np.asarray(im).reshape(img.shape)
        assert abs(_psnr(theirs, img) - p) < 1.0


def test_bad_arguments_are_refused():
    img = synth.gray(64, 48, 99)
    descs, data, infos, _ = _blocks(img, 2, 32)
    with pytest.raises(J2KError):  # block count of another geometry
        C.write_codestream(64, 48, 1, 3, descs, data, 32, 32)
    bad = descs.copy()
    bad["length"][0] = len(data) + 1
    with pytest.raises(J2KError):  # codeword beyond the bytes
        C.write_codestream(64, 48, 1, 2, bad, data, 32, 32)
    npl, lnl = _layers(descs, infos, [lambda nb: nb // 2, lambda nb: 0])
    with pytest.raises(J2KError):  # layers that shrink
        C.write_codestream(64, 48, 1, 2, descs, data, 32, 32, layers=(npl, lnl))


def test_quantiser_steps_round_trip_through_qcd():
    """Expounded steps: 5-bit exponent, 11-bit mantissa.  A step just below a power of two rounds
    up to it (the mantissa's carry goes to the exponent); every step comes back from the QCD
    within half a mantissa unit, and steps the QCD cannot hold are refused."""
    import math
    w = h = 64
    lv = 2
    n = int(L.lib().j2k_codeblock_count(w, h, lv, 32, 32))
    descs = np.zeros(n, L.CB_DESC)  # empty blocks: only the main header matters here
    data = np.zeros(1, np.uint8)
    steps = np.array([0.99999, 1.9999, 0.5, 3.0e-4, 7.5, 0.7, 100.0], np.float32)
    cs = C.write_codestream(w, h, 1, lv, descs, data, 32, 32, lossless=False, steps=steps)
    back = C.read_codestream(cs)[0]["steps"]
    for want, got in zip(steps, back):
        assert abs(float(got) - float(want)) <= float(want) * 2.0 ** -11, (want, got)
    assert float(back[0]) == 1.0 and float(back[1]) == 2.0  # carried into the exponent
    for bad in (0.0, -1.0, float("nan"), float("inf"), 1.0e-9, 1.0e6):
        st = steps.copy()
        st[3] = bad
        with pytest.raises(J2KError):
            C.write_codestream(w, h, 1, lv, descs, data, 32, 32, lossless=False, steps=st)
    # the oracle's writer encodes the same steps identically (the QCD's SPqcd fields; the guard
    # bits before them depend on the blocks)
    def spqcd(stream):
        i = stream.find(b"\xff\x5c")
        return stream[i + 5:i + 2 + int.from_bytes(stream[i + 2:i + 4], "big")]
    img = synth.gray(w, h, 3)
    assert spqcd(bytes(O.encode_image(img, lv, 32, 32, False, steps=steps))) == spqcd(cs)
    assert len(spqcd(cs)) == 2 * steps.size


def test_bit_planes_beyond_the_guard_bits_are_refused():
    """A block may not have more magnitude bit-planes than its band's exponent plus 6 (7 guard
    bits at most), or its zero bit-plane count would be negative."""
    w = h = 64
    lv = 2
    n = int(L.lib().j2k_codeblock_count(w, h, lv, 32, 32))
    descs = np.zeros(n, L.CB_DESC)
    data = np.zeros(1, np.uint8)
    descs[0]["numbps"] = 8 + 6  # LL band of a gray image: eps = 8
    C.write_codestream(w, h, 1, lv, descs, data, 32, 32)
    descs[0]["numbps"] = 8 + 7
    with pytest.raises(J2KError):
        C.write_codestream(w, h, 1, lv, descs, data, 32, 32)

