"""CPU tests of the C ABI boundary: the library loads and exports every declared symbol, and
the host-side geometry helpers agree with the oracle (no kernel is launched here)."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(j2k_[a-z0-9_]+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    import ctypes
    from roger_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    declared = _declared()
    assert declared, "no declarations found"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same set
    assert declared <= set(_lib.SIGS) | {"j2k_decoder_create/j2k_decoder_run"}


def test_version_and_status_strings():
    from roger_b200 import _lib
    L = _lib.lib()
    assert L.j2k_version() >= 1
    assert L.j2k_status_string(-5) == b"output capacity exceeded"
    # the Python table of statuses says what the library says
    for code, text in _lib.STATUS.items():
        assert L.j2k_status_string(code).decode() == text, code
    assert L.j2k_status_string(-99) == b"unknown status"


def test_every_status_entry_point_is_guarded():
    """No C++ exception crosses the C ABI: every j2k_status function the public header declares
    runs its body between J2K_API_BEGIN and J2K_API_END (one-line bodies aside)."""
    import glob
    names = set(re.findall(r"j2k_status\s+(j2k_\w+)\s*\(", open(os.path.join(ROOT, "include", "j2k_b200.h")).read()))
    found = {}
    for f in glob.glob(os.path.join(ROOT, "roger_b200", "csrc", "*.c[up]*")):
        src = open(f).read()
        for m in re.finditer(r'^(?:extern "C" )?j2k_status (j2k_\w+)\([^{;]*\{(.*?)^\}', src, re.M | re.S):
            if m.group(1) in names:
                found[m.group(1)] = m.group(2)
    assert names == set(found), sorted(names ^ set(found))
    for name, body in found.items():
        lines = [l for l in body.strip().splitlines() if l.strip()]
        assert lines[0].strip() == "J2K_API_BEGIN" and lines[-1].strip() == "J2K_API_END", name


@pytest.mark.parametrize("w,h,L,cb", [(512, 512, 5, 64), (4096, 4096, 6, 64), (33, 17, 2, 32),
                                      (1, 1, 1, 64), (2047, 65, 5, 32)])
def test_codeblock_count_matches_oracle_partition(w, h, L, cb):
    from oracle import oracle as O
    from roger_b200 import _lib
    n = 0
    for (x0, y0, sw, sh, o, lv) in O.subbands(w, h, L):
        if sw and sh:
            n += -(-sw // cb) * -(-sh // cb)
    assert _lib.lib().j2k_codeblock_count(w, h, L, cb, cb) == n


def test_invalid_arguments_are_rejected_without_a_device():
    from roger_b200 import _lib
    L = _lib.lib()
    assert L.j2k_codeblock_count(64, 64, 3, 3, 64) == 0     # not a power of two
    assert L.j2k_codeblock_count(64, 64, 3, 128, 64) == 0   # too wide
    assert L.j2k_ctx_destroy(None) == -1
    # the fused rate-distortion step: no context, no partial slots and no launch
    assert L.j2k_dwt97_rd_parts(None, 1024, 1024, 5) == 0
    assert L.j2k_dwt97_rd_forward(None, None, None, None, None, 1, 64, 64, 1, None, 0, None, None) == -1
    assert L.j2k_dwt97_rd_backward(None, None, None, None, None, 0.0, None, 1.0, None, None, 1, 64, 64, 1,
                                   None) == -1


def test_python_mirror_subbands_match_oracle():
    from oracle import oracle as O
    from roger_b200.codec import subband_rects, default_steps
    for (w, h, L) in [(512, 512, 5), (33, 17, 2), (1, 1, 3), (2047, 65, 5)]:
        assert subband_rects(w, h, L) == [tuple(s) for s in O.subbands(w, h, L)]
        assert np.array_equal(default_steps(w, h, L), O.default_steps(w, h, L))


@pytest.mark.parametrize("form", ["j2k_t1_decode_block_host", "j2k_t1_decode_block_steps_host"])
@pytest.mark.parametrize("cw,ch,orient", [(64, 64, 0), (64, 64, 1), (64, 64, 2), (64, 64, 3), (64, 4, 0),
                                          (64, 1, 3), (33, 17, 1), (8, 64, 2), (1, 1, 0)])
def test_device_decoder_logic_runs_on_host(cw, ch, orient, form):
    """The tier-1 decoder's per-block routines (the default pass / stripe / column loops and the
    one-symbol-per-step loop) are __host__ __device__; run them on the CPU against oracle-encoded
    blocks (no kernel launch)."""
    import ctypes as C
    from oracle import oracle as O
    from roger_b200 import _lib
    f = getattr(C.CDLL(_lib.LIB_PATH), form)
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_size_t]
    rng = np.random.default_rng(cw * 7 + ch + orient)
    blk = rng.laplace(0, 25, (ch, cw)).astype(np.int32)
    data, info = O.t1_encode(blk, orient)
    buf = np.frombuffer(data + b"\0", np.uint8).copy()
    out = np.zeros_like(blk)
    assert f(buf.ctypes.data, len(data), info["numbps"], info["npasses"], orient, cw, ch, out.ctypes.data, cw) == 0
    assert np.array_equal(out, blk)


@pytest.mark.parametrize("form", ["j2k_t1_decode_block_host", "j2k_t1_decode_block_steps_host"])
@pytest.mark.parametrize("cw,ch,orient", [(64, 64, 0), (64, 64, 3), (33, 17, 1), (64, 3, 2), (5, 64, 0)])
def test_device_decoder_logic_on_truncated_passes(cw, ch, orient, form):
    """The same host run of the device decoder on every pass count of oracle-encoded blocks
    (rate-control cuts end a block after any pass), against the oracle's decoder; the oracle puts
    a block cut at a plane end at the middle of its interval, the device routine leaves that to
    the kernel's sign pass."""
    import ctypes as C
    from oracle import oracle as O
    from roger_b200 import _lib
    f = getattr(C.CDLL(_lib.LIB_PATH), form)
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_size_t]
    rng = np.random.default_rng(cw * 11 + ch * 3 + orient)
    blk = (rng.laplace(0, 40, (ch, cw)) * (rng.random((ch, cw)) < 0.7)).astype(np.int32)
    data, info = O.t1_encode(blk, orient)
    nb, full = info["numbps"], info["npasses"]
    buf = np.frombuffer(data + b"\0", np.uint8).copy()
    for npasses in range(1, full + 1):
        out = np.zeros_like(blk)
        assert f(buf.ctypes.data, len(data), nb, npasses, orient, cw, ch, out.ctypes.data, cw) == 0
        half = 0
        if npasses < 3 * nb - 2 and (npasses - 1) % 3 == 0:
            plast = nb - 1 - (npasses - 1) // 3
            half = 1 << (plast - 1) if plast > 0 else 0
        got = np.where(out != 0, np.sign(out) * (np.abs(out) + half), 0)
        assert np.array_equal(got, O.t1_decode(data, nb, npasses, orient, cw, ch)), npasses
