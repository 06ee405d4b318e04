"""ctypes binding of the CPU oracle (test infrastructure only).

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
this module; the product path never imports it.  Every function takes and returns numpy arrays.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

ORDER_T800, ORDER_REF = 0, 1
STYLE_BYPASS, STYLE_RESET, STYLE_TERMALL = 1, 2, 4
MCT_NONE, MCT_RCT, MCT_ICT = 0, 1, 2
LL, HL, LH, HH = 0, 1, 2, 3


def build():
    """Compile the oracle shared library in place (gcc)."""
    import subprocess
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libj2k_oracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P, S, I, D = C.c_void_p, C.c_size_t, C.c_int, C.c_double
        sig = {
            "or_planar_fwd_i32": [P, S, S, S, I, I, P, S, S],
            "or_planar_fwd_f32": [P, S, S, S, I, I, P, S, S],
            "or_planar_inv_i32": [P, S, S, S, S, I, I, P, S],
            "or_planar_inv_f32": [P, S, S, S, S, I, I, P, S],
            "or_dwt53_fwd": [P, S, P, S, S, S, I, I],
            "or_dwt53_inv": [P, S, P, S, S, S, I, I],
            "or_dwt97_fwd_f32": [P, S, P, S, S, S, I, I],
            "or_dwt97_inv_f32": [P, S, P, S, S, S, I, I],
            "or_dwt97_fwd_f64": [P, S, P, S, S, S, I, I],
            "or_dwt97_inv_f64": [P, S, P, S, S, S, I, I],
            "or_dwt97_fwd_adj_f64": [P, S, P, S, S, S, I],
            "or_dwt97_inv_adj_f64": [P, S, P, S, S, S, I],
            "or_subband_rect": [S, S, I, I, P, P, P, P, P, P],
            "or_quantize_f32": [P, S, P, S, S, S, I, P],
            "or_dequantize_f32": [P, S, P, S, S, S, I, P],
            "or_t1_encode": [P, S, I, I, I, P, I, P, I, P],
            "or_t1_decode": [P, I, I, I, I, P, S, I, I],
            "or_t1_encode_styled": [P, S, I, I, I, I, P, I, P, P],
            "or_t1_decode_styled": [P, I, P, I, I, I, I, P, S, I, I],
            "or_t1_pass_raw": [I, I],
            "or_t1_pass_terminated": [I, I, I],
            "or_encode_image": [P, S, S, I, P, P, C.c_long],
            "or_philox_uniform": [C.c_uint64, C.c_uint64],
            "or_rd_noise": [C.c_uint64, S, S, S],
            "or_t1_plane_distortion": [P, S, I, I, I, P],
            "or_rd_loss_f64": [P, S, S, I, P, D, C.c_uint64, P, P],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
        L.or_t1_encode.restype = I
        L.or_t1_decode.restype = I
        L.or_t1_encode_styled.restype = I
        L.or_t1_decode_styled.restype = I
        L.or_t1_pass_raw.restype = I
        L.or_t1_pass_terminated.restype = I
        L.or_subband_rect.restype = I
        L.or_encode_image.restype = C.c_long
        L.or_philox_uniform.restype = D
        L.or_rd_noise.restype = D
        L.or_rd_loss_f64.restype = D
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class T1Info(C.Structure):
    _fields_ = [("numbps", C.c_int), ("npasses", C.c_int), ("length", C.c_int), ("nsyms", C.c_int),
                ("plane_bytes", C.c_int * 32)]


class EncParams(C.Structure):
    _fields_ = [("levels", C.c_int), ("cbw", C.c_int), ("cbh", C.c_int), ("lossless", C.c_int),
                ("order", C.c_int), ("steps", C.c_void_p), ("tier1_only", C.c_int), ("style", C.c_int)]


def planar_fwd(img, mct, as_float=False):
    """img: (h, w, ncomp) or (h, w) uint8 -> (ncomp, h, w) int32 or float32 planes."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    if img.ndim == 2:
        img = img[:, :, None]
    h, w, nc = img.shape
    out = np.empty((nc, h, w), np.float32 if as_float else np.int32)
    fn = lib().or_planar_fwd_f32 if as_float else lib().or_planar_fwd_i32
    fn(_p(img), w, h, w * nc, nc, mct, _p(out), w, w * h)
    return out


def planar_inv(planes, mct):
    planes = np.ascontiguousarray(planes)
    nc, h, w = planes.shape
    out = np.empty((h, w, nc), np.uint8)
    if planes.dtype == np.int32:
        lib().or_planar_inv_i32(_p(planes), w, w * h, w, h, nc, mct, _p(out), w * nc)
    else:
        planes = planes.astype(np.float32)
        lib().or_planar_inv_f32(_p(planes), w, w * h, w, h, nc, mct, _p(out), w * nc)
    return out


def _dwt(fn, a, dtype, levels, order=None):
    a = np.ascontiguousarray(a, dtype=dtype)
    h, w = a.shape
    out = np.empty_like(a)
    if order is None:
        fn(_p(a), w, _p(out), w, w, h, levels)
    else:
        fn(_p(a), w, _p(out), w, w, h, levels, order)
    return out


def dwt53_fwd(a, levels, order=ORDER_T800):
    return _dwt(lib().or_dwt53_fwd, a, np.int32, levels, order)


def dwt53_inv(a, levels, order=ORDER_T800):
    return _dwt(lib().or_dwt53_inv, a, np.int32, levels, order)


def dwt97_fwd(a, levels, order=ORDER_T800, f64=False):
    fn = lib().or_dwt97_fwd_f64 if f64 else lib().or_dwt97_fwd_f32
    return _dwt(fn, a, np.float64 if f64 else np.float32, levels, order)


def dwt97_inv(a, levels, order=ORDER_T800, f64=False):
    fn = lib().or_dwt97_inv_f64 if f64 else lib().or_dwt97_inv_f32
    return _dwt(fn, a, np.float64 if f64 else np.float32, levels, order)


def dwt97_fwd_adj(g, levels):
    return _dwt(lib().or_dwt97_fwd_adj_f64, g, np.float64, levels)


def dwt97_inv_adj(g, levels):
    return _dwt(lib().or_dwt97_inv_adj_f64, g, np.float64, levels)


def subbands(w, h, levels):
    """List of (x0, y0, sw, sh, orient, level) in T.800 QCD order."""
    res = []
    v = [C.c_size_t() for _ in range(4)]
    o, lv = C.c_int(), C.c_int()
    for b in range(3 * levels + 1):
        lib().or_subband_rect(w, h, levels, b, *[C.byref(x) for x in v], C.byref(o), C.byref(lv))
        res.append((v[0].value, v[1].value, v[2].value, v[3].value, o.value, lv.value))
    return res


def default_steps(w, h, levels):
    """Per-subband step 8*2^-k, k = decomposition level of the subband."""
    return np.array([8.0 * 2.0 ** -sb[5] for sb in subbands(w, h, levels)], np.float32)


def quantize(coef, levels, steps):
    coef = np.ascontiguousarray(coef, np.float32)
    h, w = coef.shape
    q = np.empty((h, w), np.int32)
    steps = np.ascontiguousarray(steps, np.float32)
    lib().or_quantize_f32(_p(coef), w, _p(q), w, w, h, levels, _p(steps))
    return q


def dequantize(q, levels, steps):
    q = np.ascontiguousarray(q, np.int32)
    h, w = q.shape
    out = np.empty((h, w), np.float32)
    steps = np.ascontiguousarray(steps, np.float32)
    lib().or_dequantize_f32(_p(q), w, _p(out), w, w, h, levels, _p(steps))
    return out


def t1_encode(block, orient, want_symbols=False):
    """Encodes one code-block (2-D int32).  Returns (bytes, info dict[, symbols])."""
    block = np.ascontiguousarray(block, np.int32)
    ch, cw = block.shape
    cap = cw * ch * 8 + 256
    out = np.empty(cap, np.uint8)
    info = T1Info()
    scap = cw * ch * 70 + 64 if want_symbols else 0
    syms = np.empty(max(scap, 1), np.uint8) if want_symbols else None
    n = lib().or_t1_encode(_p(block), cw, cw, ch, orient, _p(out), cap, _p(syms), scap,
                           C.byref(info))
    if n < 0:
        raise RuntimeError("oracle t1 encode overflow")
    d = dict(numbps=info.numbps, npasses=info.npasses, length=info.length, nsyms=info.nsyms,
             plane_bytes=list(info.plane_bytes[:info.numbps]))
    if want_symbols:
        return out[:n].tobytes(), d, syms[:info.nsyms].copy()
    return out[:n].tobytes(), d


def t1_encode_styled(block, orient, style):
    """Encodes one code-block with a code-block style.  Returns (bytes, info dict, pass_end
    list: codeword bytes at the end of each pass, exact where the pass is terminated)."""
    block = np.ascontiguousarray(block, np.int32)
    ch, cw = block.shape
    cap = cw * ch * 8 + 1024
    out = np.empty(cap, np.uint8)
    info = T1Info()
    pe = np.zeros(96, np.int32)
    n = lib().or_t1_encode_styled(_p(block), cw, cw, ch, orient, style, _p(out), cap, C.byref(info), _p(pe))
    if n < 0:
        raise RuntimeError("oracle t1 encode overflow")
    d = dict(numbps=info.numbps, npasses=info.npasses, length=info.length, nsyms=info.nsyms)
    return out[:n].tobytes(), d, [int(v) for v in pe[:info.npasses]]


def t1_decode_styled(data, pass_end, numbps, npasses, orient, cw, ch, style):
    buf = np.frombuffer(bytes(data) + b"\0", np.uint8).copy()
    pe = np.ascontiguousarray(np.asarray(pass_end, np.int32)) if pass_end is not None else None
    out = np.empty((ch, cw), np.int32)
    r = lib().or_t1_decode_styled(_p(buf), len(data), _p(pe), numbps, npasses, orient, style, _p(out), cw, cw, ch)
    if r != 0:
        raise RuntimeError("oracle t1 decode failed")
    return out


def pass_raw(style, p):
    return bool(lib().or_t1_pass_raw(style, p))


def pass_terminated(style, p, npasses):
    return bool(lib().or_t1_pass_terminated(style, p, npasses))


def t1_decode(data, numbps, npasses, orient, cw, ch):
    buf = np.frombuffer(bytes(data) + b"\0", np.uint8).copy()
    out = np.empty((ch, cw), np.int32)
    r = lib().or_t1_decode(_p(buf), len(data), numbps, npasses, orient, _p(out), cw, cw, ch)
    if r != 0:
        raise RuntimeError("oracle t1 decode failed")
    return out


def encode_tier1(img, levels, cbw=64, cbh=64, lossless=True, order=ORDER_T800, steps=None, style=0):
    """Whole-image oracle encode up to the code-blocks' codewords (planar, colour transform,
    DWT, quantiser, tier-1; no tier-2) -> the sum of the codeword lengths."""
    img = np.ascontiguousarray(img, np.uint8)
    if img.ndim == 2:
        img = img[:, :, None]
    h, w, nc = img.shape
    st = None if steps is None else np.ascontiguousarray(steps, np.float32)
    par = EncParams(levels, cbw, cbh, int(lossless), order, st.ctypes.data if st is not None else None, 1, style)
    n = lib().or_encode_image(_p(img), w, h, nc, C.byref(par), None, 0)
    if n < 0:
        raise RuntimeError("oracle tier-1 encode failed")
    return int(n)


def encode_image(img, levels, cbw=64, cbh=64, lossless=True, order=ORDER_T800, steps=None, style=0):
    """Whole-image oracle encoder -> raw J2K codestream bytes (style: code-block style bits,
    STYLE_*)."""
    img = np.ascontiguousarray(img, np.uint8)
    if img.ndim == 2:
        img = img[:, :, None]
    h, w, nc = img.shape
    st = None if steps is None else np.ascontiguousarray(steps, np.float32)
    par = EncParams(levels, cbw, cbh, int(lossless), order, st.ctypes.data if st is not None else None, 0, style)
    cap = w * h * nc * 4 + 65536
    out = np.empty(cap, np.uint8)
    n = lib().or_encode_image(_p(img), w, h, nc, C.byref(par), _p(out), cap)
    if n < 0:
        raise RuntimeError("oracle codestream overflow")
    return out[:n].tobytes()


def philox_uniform(seed, i):
    return lib().or_philox_uniform(seed, i)


def rd_noise(seed, w, x, y):
    """Noise sample of the relaxed quantiser at Mallat position (x, y) of a w-wide plane."""
    return lib().or_rd_noise(seed, w, x, y)


def rd_loss(x, levels, log_steps, lam, seed, grads=True):
    x = np.ascontiguousarray(x, np.float64)
    h, w = x.shape
    ls = np.ascontiguousarray(log_steps, np.float64)
    gx = np.empty_like(x) if grads else None
    gl = np.empty_like(ls) if grads else None
    loss = lib().or_rd_loss_f64(_p(x), w, h, levels, _p(ls), lam, seed, _p(gx), _p(gl))
    return (loss, gx, gl) if grads else loss


TRUNC_EXTRA = 4


def truncation_length(info, k):
    """Codeword bytes kept when the block is cut after bit-plane k (npasses = 3k+1)."""
    if k >= info["numbps"] - 1:
        return info["length"]
    return min(info["length"], info["plane_bytes"][k] + TRUNC_EXTRA)


def plane_distortion(block, numbps):
    block = np.ascontiguousarray(block, np.int32)
    ch, cw = block.shape
    out = np.zeros(33, np.float64)
    lib().or_t1_plane_distortion(_p(block), cw, cw, ch, numbps, _p(out))
    return out
