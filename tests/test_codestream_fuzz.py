"""Robustness of the host tier-2 reader (j2k_codestream_info / j2k_codestream_read_layers), on
the CPU: truncated and corrupted codestreams either parse into self-consistent descriptors or
are refused with a status and a reason; nothing crashes and no exception crosses the C ABI.
Mutated headers that claim more than a million code-blocks are only sized, not parsed: a header
may legitimately describe a huge image, and empty packets cost no bytes per block."""
import io

import numpy as np
import pytest

from oracle import oracle as O
from roger_b200 import codec as C
from roger_b200 import synth
from roger_b200._lib import J2KError

PIL = pytest.importorskip("PIL.Image")


def _streams():
    out = [bytes(O.encode_image(synth.rgb(96, 80, (5, 6, 7, 8)), 3, 32, 32, True)),
           bytes(O.encode_image(synth.gray(131, 97, 9), 4, 64, 64, True))]
    buf = io.BytesIO()
    PIL.fromarray(synth.rgb(72, 56, (11, 12, 13, 14))).save(
        buf, "JPEG2000", irreversible=False, mct=1, num_resolutions=4, codeblock_size=(16, 16), progression="RLCP",
        quality_mode="rates", quality_layers=[40, 10, 1], no_jp2=True)
    out.append(buf.getvalue())
    return out


def _check(cs):
    try:
        info = C.codestream_info(cs)
    except J2KError as e:
        assert e.status < 0 and str(e)
        return "refused"
    nblk = sum(-(-info["w"] // info["cbw"]) * -(-info["h"] // info["cbh"]) for _ in range(info["ncomp"]))
    if nblk > 1 << 20:
        return "huge"
    try:
        d, descs, data = C.read_codestream(cs)
    except J2KError as e:
        assert e.status < 0 and str(e)
        return "refused"
    assert d["w"] == info["w"] and d["h"] == info["h"] and d["ncomp"] == info["ncomp"]
    ln = descs["length"].astype(np.int64)
    assert (ln >= 0).all()
    assert (descs["offset"].astype(np.int64) + ln <= data.size).all()
    assert (descs["numbps"] <= 31).all()
    assert (descs["npasses"].astype(np.int64) <= 3 * descs["numbps"].astype(np.int64)).all()
    return "parsed"


@pytest.mark.parametrize("which", [0, 1, 2])
def test_truncated_and_corrupted_streams_are_parsed_or_refused(which):
    cs = _streams()[which]
    assert _check(cs) == "parsed"
    rng = np.random.default_rng(1000 + which)
    seen = {"parsed": 0, "refused": 0, "huge": 0}
    for n in sorted(set(rng.integers(0, len(cs), 60).tolist())) + [0, 1, 2, len(cs) - 1]:
        seen[_check(cs[:n])] += 1
    for _ in range(300):
        m = bytearray(cs)
        for _ in range(int(rng.integers(1, 5))):
            # headers (the first 200 bytes) are hit as often as the packets
            hi = min(len(m), 200) if rng.random() < 0.5 else len(m)
            k = int(rng.integers(0, hi))
            kind = rng.random()
            if kind < 0.6:
                m[k] = int(rng.integers(0, 256))
            elif kind < 0.8:
                m[k] = 0xFF
            else:
                del m[k:k + int(rng.integers(1, 9))]
        seen[_check(bytes(m))] += 1
    assert seen["refused"] > 0 and seen["parsed"] > 0
