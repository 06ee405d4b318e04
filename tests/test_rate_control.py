"""Rate control (PCRD-opt truncation of the code-blocks to a byte budget, one quality layer).

CPU: the truncation rule (bytes produced at the end of a bit-plane + 4) decodes every kept pass
exactly as the whole codeword does, and the per-plane distortions behave.  GPU: codestreams cut
to a target are within it, decode through OpenJPEG and through this library's GPU decoder,
whose output is identical to the oracle's decode of the same codestream, and quality rises with
the budget up to lossless."""
import io

import numpy as np
import pytest

from oracle import oracle as O
from roger_b200 import synth


def _blocks(img, L, cb):
    co = O.dwt53_fwd(img.astype(np.int32) - 128, L)
    h, w = img.shape
    for (x0, y0, sw, sh, o, lv) in O.subbands(w, h, L):
        for by in range(y0, y0 + sh, cb):
            for bx in range(x0, x0 + sw, cb):
                yield o, co[by:min(by + cb, y0 + sh), bx:min(bx + cb, x0 + sw)]


def test_truncated_codewords_decode_like_whole_ones():
    img = synth.gray(192, 160, 7)
    n = 0
    for o, blk in _blocks(img, 4, 32):
        data, info = O.t1_encode(blk, o)
        nb = info["numbps"]
        for k in range(nb):
            L = O.truncation_length(info, k)
            assert L <= info["length"]
            a = O.t1_decode(data[:L], nb, 3 * k + 1, o, blk.shape[1], blk.shape[0])
            b = O.t1_decode(data, nb, 3 * k + 1, o, blk.shape[1], blk.shape[0])
            assert np.array_equal(a, b)
            n += 1
    assert n > 100


def test_plane_distortion_decreases_to_zero():
    img = synth.gray(128, 128, 8)
    for o, blk in _blocks(img, 3, 32):
        data, info = O.t1_encode(blk, o)
        nb = info["numbps"]
        d = O.plane_distortion(blk, nb)
        assert d[32] == float((blk.astype(np.float64) ** 2).sum())
        if nb:
            assert all(d[k + 1] <= d[k] for k in range(nb - 1))
            assert d[0] <= d[32] and d[nb - 1] == 0.0


def _psnr(a, b):
    e = a.astype(np.float64) - b.astype(np.float64)
    mse = float((e * e).mean())
    return float("inf") if mse == 0 else 10 * np.log10(255.0 ** 2 / mse)


def _oracle_decode(cs):
    from roger_b200 import codec as C
    info, descs, data = C.read_codestream(cs)
    w, h, nc, L = info["w"], info["h"], info["ncomp"], info["levels"]
    planes = np.zeros((nc, h, w), np.int32)
    for d in descs:
        if d["npasses"] == 0:
            continue
        blk = O.t1_decode(bytes(data[d["offset"]:d["offset"] + d["length"]]), int(d["numbps"]),
                          int(d["npasses"]), int(d["orient"]), int(d["cw"]), int(d["ch"]))
        planes[d["comp"], d["y0"]:d["y0"] + d["ch"], d["x0"]:d["x0"] + d["cw"]] = blk
    rec = np.stack([O.dwt53_inv(p, L) for p in planes])
    return O.planar_inv(rec, 1 if nc == 3 else 0).reshape(h, w, nc)


@pytest.mark.gpu
def test_rate_controlled_codestreams():
    from PIL import Image
    from roger_b200 import codec as C
    img = synth.rgb(384, 256, (31, 32, 33, 34))
    enc = C.OCLEncoder(lossy=False)
    full = len(enc.run_rgb(img, levels=5, cbw=32, cbh=32).codestream())
    last = -1.0
    for frac in (0.03, 0.1, 0.3, 0.6):
        target = int(full * frac)
        cs = bytes(enc.run_rgb(img, levels=5, cbw=32, cbh=32, target_bytes=target).codestream())
        assert 0.8 * target <= len(cs) <= target
        ours = C.decode_codestream(cs).reshape(img.shape)
        assert np.array_equal(ours, _oracle_decode(cs).reshape(img.shape))
        theirs = np.asarray(Image.open(io.BytesIO(cs))).reshape(img.shape)
        p_ours, p_theirs = _psnr(ours, img), _psnr(theirs, img)
        assert p_ours > last and abs(p_ours - p_theirs) < 1.0
        last = p_ours
    cs = bytes(enc.run_rgb(img, levels=5, cbw=32, cbh=32, target_bytes=10 * full).codestream())
    assert np.array_equal(C.decode_codestream(cs).reshape(img.shape), img)


def _pcrd_reference(desc, pb, dist, w, budget, extra=4):
    """Plain restatement of the truncation choice: convex hulls, then the hull segments in order
    of decreasing slope are kept until the first that does not fit; that slope and lower go."""
    hulls = []
    for i, d in enumerate(desc):
        nb, npas, ln = int(d["numbps"]), int(d["npasses"]), int(d["length"])
        pts = [(0.0, dist[i, 32] * w[i], 0)]
        for k in range(min(nb, 31)):
            np_ = 3 * k + 1
            if np_ > npas:
                break
            L = float(ln) if k == nb - 1 else min(float(ln), float(pb[i, k]) + extra)
            L = max(L, pts[-1][0])  # a later cut never keeps fewer bytes
            pts.append((L, dist[i, k] * w[i], np_))
        h = []
        for p in pts:
            if h and p[0] <= h[-1][0]:
                if p[1] < h[-1][1]:
                    h[-1] = p
                continue
            if h and p[1] >= h[-1][1]:
                continue
            while len(h) >= 2:
                a, b = h[-2], h[-1]
                if (b[1] - p[1]) * (b[0] - a[0]) >= (a[1] - b[1]) * (p[0] - b[0]):
                    h.pop()
                else:
                    break
            h.append(p)
        hulls.append(h)
    segs = sorted(((h[q - 1][1] - h[q][1]) / (h[q][0] - h[q - 1][0]), h[q][0] - h[q - 1][0])
                  for h in hulls for q in range(1, len(h)))[::-1]
    thr, room = -1.0, float(budget)
    if sum(s[1] for s in segs) > budget:
        for s, dl in segs:
            if dl > room:
                thr = s
                break
            room -= dl
    out = []
    for h in hulls:
        q = 0
        while q + 1 < len(h) and (h[q][1] - h[q + 1][1]) / (h[q + 1][0] - h[q][0]) > thr:
            q += 1
        out.append((h[q][2], int(h[q][0]) if h[q][2] else 0))
    return out


@pytest.mark.parametrize("seed,n", [(1, 700), (2, 700), (3, 6000)])
def test_pcrd_selection_matches_sorted_threshold(seed, n):
    """n = 6000 builds the blocks' hulls on several host threads (4096 blocks and more)."""
    import ctypes as C
    from roger_b200 import _lib
    f = C.CDLL(_lib.LIB_PATH).j2k_pcrd_truncate
    f.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]
    f.restype = C.c_int
    rng = np.random.default_rng(seed)
    desc = np.zeros(n, _lib.CB_DESC)
    pb = np.zeros((n, 32), np.uint32)
    dist = np.zeros((n, 33))
    for i in range(n):
        nb = int(rng.integers(0, 14))
        desc[i]["numbps"] = nb
        desc[i]["npasses"] = max(3 * nb - 2, 0)
        steps = rng.integers(0, 400, nb)
        cum = np.cumsum(steps)
        pb[i, :nb] = cum
        desc[i]["length"] = int(cum[-1]) + 3 if nb else 0
        d = np.sort(rng.exponential(1e6, nb + 1))[::-1]
        d[-1] = 0.0
        dist[i, 32] = d[0] if nb else 0.0
        dist[i, :nb] = d[1:]
        if nb and rng.random() < 0.1:  # a plane that adds bytes but lowers nothing
            k = int(rng.integers(0, nb))
            dist[i, k] = dist[i, 32] if k == 0 else dist[i, k - 1]
    w = rng.uniform(0.1, 3.0, n)
    full = int(desc["length"].sum())
    for frac in (0.0, 0.05, 0.3, 0.8, 1.2):
        budget = int(full * frac)
        d2 = desc.copy()
        assert f(d2.ctypes.data, n, pb.ctypes.data, dist.ctypes.data, w.ctypes.data, budget) == 0
        ref = _pcrd_reference(desc, pb, dist, w, budget)
        assert [(int(a), int(b)) for a, b in zip(d2["npasses"], d2["length"])] == ref
        assert int(d2["length"].sum()) <= min(budget, full)


def test_pcrd_ties_drop_together():
    """Thousands of identical blocks give hull segments of equal slope; a budget that falls inside
    such a group drops the whole group, as the sorted restatement does (threaded hull build)."""
    import ctypes as C
    from roger_b200 import _lib
    f = C.CDLL(_lib.LIB_PATH).j2k_pcrd_truncate
    f.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]
    f.restype = C.c_int
    n = 5000
    desc = np.zeros(n, _lib.CB_DESC)
    pb = np.zeros((n, 32), np.uint32)
    dist = np.zeros((n, 33))
    kinds = [(5, [40, 90, 200, 420, 800], [6e5, 2e5, 5e4, 9e3, 0.0], 1e6),
             (3, [10, 60, 300], [3e5, 4e4, 0.0], 8e5)]
    for i in range(n):
        nb, cum, d, d0 = kinds[i % 3 == 0]
        desc[i]["numbps"] = nb
        desc[i]["npasses"] = 3 * nb - 2
        desc[i]["length"] = cum[-1] + 3
        pb[i, :nb] = cum
        dist[i, 32] = d0
        dist[i, :nb] = d
    w = np.where(np.arange(n) % 2 == 0, 1.0, 2.0)  # two bands: ties within each
    full = int(desc["length"].sum())
    for frac in (0.01, 0.1, 0.25, 0.5, 0.75, 0.99):
        budget = int(full * frac)
        d2 = desc.copy()
        assert f(d2.ctypes.data, n, pb.ctypes.data, dist.ctypes.data, w.ctypes.data, budget) == 0
        ref = _pcrd_reference(desc, pb, dist, w, budget)
        assert [(int(a), int(b)) for a, b in zip(d2["npasses"], d2["length"])] == ref
        assert int(d2["length"].sum()) <= budget


def test_pcrd_holds_the_budget_for_any_plane_positions():
    """Plane-end byte positions that do not increase (never produced by the coder) are held
    non-decreasing, so the cut still fits the budget and matches the restatement."""
    import ctypes as C
    from roger_b200 import _lib
    f = C.CDLL(_lib.LIB_PATH).j2k_pcrd_truncate
    f.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]
    f.restype = C.c_int
    rng = np.random.default_rng(11)
    n = 500
    desc = np.zeros(n, _lib.CB_DESC)
    nb = rng.integers(1, 12, n)
    desc["numbps"] = nb
    desc["npasses"] = 3 * nb - 2
    desc["length"] = rng.integers(100, 3000, n)
    pb = rng.integers(0, 3000, (n, 32)).astype(np.uint32)  # in no particular order
    dist = np.sort(rng.exponential(1e6, (n, 33)), axis=1)[:, ::-1]
    dist = np.ascontiguousarray(np.concatenate([dist[:, 1:], dist[:, :1]], axis=1))  # [32]: nothing decoded
    w = rng.uniform(0.5, 2.0, n)
    full = int(desc["length"].sum())
    for frac in (0.05, 0.2, 0.5, 0.9):
        budget = int(full * frac)
        d2 = desc.copy()
        assert f(d2.ctypes.data, n, pb.ctypes.data, dist.ctypes.data, w.ctypes.data, budget) == 0
        assert int(d2["length"].sum()) <= budget
        assert [(int(a), int(b)) for a, b in zip(d2["npasses"], d2["length"])] == _pcrd_reference(desc, pb, dist, w, budget)


@pytest.mark.gpu
def test_quality_layers():
    from PIL import Image
    from roger_b200 import codec as C
    img = synth.rgb(384, 256, (51, 52, 53, 54))
    enc = C.OCLEncoder(lossy=False)
    full = len(enc.run_rgb(img, levels=5, cbw=32, cbh=32).codestream())
    budgets = [int(full * 0.04), int(full * 0.15), int(full * 0.4), 0]
    single = bytes(enc.run_rgb(img, levels=5, cbw=32, cbh=32, target_bytes=budgets[0]).codestream())
    cs = bytes(enc.run_rgb(img, levels=5, cbw=32, cbh=32, layers=budgets).codestream())
    info, descs, _ = C.read_codestream(cs)
    assert info["layers"] == 4
    # the last layer keeps every pass: lossless for us and for OpenJPEG
    assert np.array_equal(C.decode_codestream(cs).reshape(img.shape), img)
    assert np.array_equal(np.asarray(Image.open(io.BytesIO(cs))).reshape(img.shape), img)
    # layer 0 is the single-layer cut at the same budget, block by block
    _, d1, b1 = C.read_codestream(single)
    _, d0, b0 = C.read_codestream(cs, max_layers=1)
    assert np.array_equal(d0["npasses"], d1["npasses"]) and np.array_equal(d0["length"], d1["length"])
    assert np.array_equal(b0, b1)
    # every prefix of layers: codeword bytes within its budget, quality rising, GPU decode equal
    # to the oracle's and close to OpenJPEG's decode of the same layers
    last = -1.0
    for k in (1, 2, 3):
        _, dk, _ = C.read_codestream(cs, max_layers=k)
        assert int(dk["length"].sum()) <= budgets[k - 1]
        ours = C.decode_codestream(cs, max_layers=k).reshape(img.shape)
        p = _psnr(ours, img)
        assert p > last
        last = p
        im = Image.open(io.BytesIO(cs))
        t = im.tile[0]
        im.tile = [type(t)(t[0], t[1], t[2], (t[3][0], 0, k) + tuple(t[3][3:]))]
        theirs = np.asarray(im).reshape(img.shape)
        assert abs(_psnr(theirs, img) - p) < 1.0


@pytest.mark.gpu
def test_rate_control_never_exceeds_the_budget():
    from roger_b200 import codec as C
    img = synth.rgb(512, 384, (75, 76, 77, 78))
    enc = C.OCLEncoder()
    for t in list(range(11900, 12101, 13)) + [2500, 5000, 20000, 40000]:
        n = len(bytes(enc.run_rgb(img, levels=5, target_bytes=t).codestream()))
        assert n <= t, (t, n)


@pytest.mark.gpu
def test_cut_lengths_are_the_oracles_plane_end_lengths():
    # every cut block keeps exactly the bytes the oracle's MQ coder had produced at the end of
    # that bit-plane, plus the read-ahead margin: checks the rate pass's plane-end records
    from roger_b200 import codec as C
    img = synth.rgb(256, 192, (81, 82, 83, 84))
    L = 4
    enc = C.OCLEncoder()
    full = len(enc.run_rgb(img, levels=L, cbw=32, cbh=32).codestream())
    planes = O.planar_fwd(img, 1)
    coef = [O.dwt53_fwd(planes[c], L) for c in range(3)]
    checked = 0
    for frac in (0.05, 0.2, 0.5):
        cs = bytes(enc.run_rgb(img, levels=L, cbw=32, cbh=32, target_bytes=int(full * frac)).codestream())
        _, descs, _ = C.read_codestream(cs)
        for d in descs:
            if d["npasses"] == 0:
                continue
            blk = coef[d["comp"]][d["y0"]:d["y0"] + d["ch"], d["x0"]:d["x0"] + d["cw"]]
            _, info = O.t1_encode(blk, int(d["orient"]))
            assert info["numbps"] == d["numbps"]
            k = (int(d["npasses"]) - 1) // 3
            assert (int(d["npasses"]) - 1) % 3 == 0
            assert int(d["length"]) == O.truncation_length(info, k)
            checked += 1
    assert checked > 100
