"""Python mirror of the reference's operator interface, over the C ABI of libj2kb200.

Class and method names follow knopkem/roger (src/OCLEncoder.h:27-37, src/OCLDecoder.h:25-34,
src/OCLDWTForward.h:31, src/OCLDWTRev.h:31, src/OCLRGBtoPlanar.h:28, src/OCLBPC.h:28,
src/OCLEncodeDecode.h:23-38).  Device buffers are torch CUDA tensors (torch is used for device
memory and streams only; every computation runs in the library's CUDA kernels).  Errors raise
J2KError instead of being logged and swallowed as the reference's LogError did.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib as L
from ._lib import J2KError, check, lib

__all__ = ["Context", "rgb_to_planar", "planar_to_rgb", "dwt_forward", "dwt_inverse",
           "codeblock_count", "bpc_encode", "bpc_decode", "OCLEncoder", "OCLDecoder",
           "OCLDWTForward", "OCLDWTRev", "OCLRGBtoPlanar", "OCLBPC", "default_steps", "read_codestream",
           "decode_codestream",
           "read_pass_ends", "subband_rects", "J2KError"]


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def subband_rects(w, h, levels):
    """[(x0, y0, sw, sh, orient, level)] in T.800 QCD order (LL_L, then HL/LH/HH for L..1)."""
    ws, hs = [w], [h]
    for _ in range(levels):
        ws.append((ws[-1] + 1) // 2)
        hs.append((hs[-1] + 1) // 2)
    out = [(0, 0, ws[levels], hs[levels], L.BAND_LL, levels)]
    for k in range(levels, 0, -1):
        lw, lh, pw, ph = ws[k], hs[k], ws[k - 1], hs[k - 1]
        out.append((lw, 0, pw - lw, lh, L.BAND_HL, k))
        out.append((0, lh, lw, ph - lh, L.BAND_LH, k))
        out.append((lw, lh, pw - lw, ph - lh, L.BAND_HH, k))
    return out


def default_steps(w, h, levels):
    """Dead-zone quantiser steps 8 * 2^-k for a subband of decomposition level k."""
    return np.array([8.0 * 2.0 ** -sb[5] for sb in subband_rects(w, h, levels)], np.float32)


class Context:
    """Device context (replaces OCLDeviceManager + ocl_args_d_t + the in-order OCLQueue).

    By default the context follows torch's current CUDA stream so that its launches order
    with torch tensor operations."""

    def __init__(self, device=0, use_torch_stream=True):
        self.device = device
        h = C.c_void_p()
        check(lib().j2k_ctx_create(device, C.byref(h)))
        self.h = h
        self.use_torch_stream = use_torch_stream

    def _bind(self):
        if self.use_torch_stream:
            s = torch.cuda.current_stream(self.device).cuda_stream
            check(lib().j2k_ctx_set_stream(self.h, C.c_void_p(s)), self.h)
        return self.h

    def sync(self):
        check(lib().j2k_stream_sync(self.h), self.h)

    def close(self):
        if self.h:
            lib().j2k_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_DEFAULT = {}


def default_context(device=0):
    if device not in _DEFAULT:
        _DEFAULT[device] = Context(device)
    return _DEFAULT[device]


def _dtype_code(t):
    return {torch.int32: L.I32, torch.float32: L.F32, torch.uint8: L.U8, torch.int16: L.I16}[t.dtype]


def _need_cuda(t, name):
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise TypeError(f"{name} must be a CUDA tensor")


def rgb_to_planar(img, mct=L.MCT_RCT, ctx=None, out_dtype=None):
    """img: (H, W, C) or (H, W) uint8 CUDA tensor -> (C, H, W) int32 (RCT/none) or float32 (ICT)."""
    ctx = ctx or default_context(img.device.index or 0)
    _need_cuda(img, "img")
    if img.dim() == 2:
        img = img.unsqueeze(-1)
    img = img.contiguous()
    h, w, nc = img.shape
    if out_dtype is None:
        out_dtype = torch.float32 if mct == L.MCT_ICT else torch.int32
    planes = torch.empty((nc, h, w), dtype=out_dtype, device=img.device)
    hh = ctx._bind()
    check(lib().j2k_rgb_to_planar(hh, _ptr(img), w * nc, nc, mct, _dtype_code(planes), _ptr(planes),
                                  w, w * h, w, h), hh)
    return planes


def planar_to_rgb(planes, mct=L.MCT_RCT, ctx=None):
    ctx = ctx or default_context(planes.device.index or 0)
    _need_cuda(planes, "planes")
    planes = planes.contiguous()
    nc, h, w = planes.shape
    out = torch.empty((h, w, nc), dtype=torch.uint8, device=planes.device)
    hh = ctx._bind()
    check(lib().j2k_planar_to_rgb(hh, _ptr(planes), _dtype_code(planes), w, w * h, nc, mct,
                                  _ptr(out), w * nc, w, h), hh)
    return out


def _steps_arg(steps, levels):
    if steps is None:
        return None, None
    a = np.ascontiguousarray(steps, np.float32)
    if a.size != 3 * levels + 1:
        raise ValueError(f"need {3 * levels + 1} steps, got {a.size}")
    return a, a.ctypes.data_as(C.c_void_p)


def dwt_forward(plane, levels, kernel=None, order=L.ORDER_T800, steps=None, ctx=None, out=None):
    """Forward DWT of one (H, W) plane or a batch (N, H, W) of planes (int32 -> 5/3,
    float32 -> 9/7), Mallat output.  With steps (9/7 only) the output is int32 dead-zone
    indices.  A batch is transformed with one launch per level."""
    ctx = ctx or default_context(plane.device.index or 0)
    _need_cuda(plane, "plane")
    if kernel is None:
        kernel = L.W53 if plane.dtype == torch.int32 else L.W97
    h, w = plane.shape[-2:]
    odt = torch.int32 if (kernel == L.W53 or steps is not None) else torch.float32
    if out is None:
        out = torch.empty(plane.shape, dtype=odt, device=plane.device)
    keep, sp = _steps_arg(steps, levels)
    hh = ctx._bind()
    if plane.dim() == 3:
        check(lib().j2k_dwt_forward_batch(hh, kernel, order, _ptr(plane), plane.stride(1), plane.stride(0),
                                          _ptr(out), out.stride(1), out.stride(0), plane.shape[0], w, h,
                                          levels, sp), hh)
    else:
        check(lib().j2k_dwt_forward(hh, kernel, order, _ptr(plane), plane.stride(0), _ptr(out),
                                    out.stride(0), w, h, levels, sp), hh)
    return out


def dwt_inverse(coef, levels, kernel=None, order=L.ORDER_T800, steps=None, ctx=None, out=None):
    """Inverse DWT of one (H, W) Mallat plane or a batch (N, H, W)."""
    ctx = ctx or default_context(coef.device.index or 0)
    _need_cuda(coef, "coef")
    if kernel is None:
        kernel = L.W53 if (coef.dtype == torch.int32 and steps is None) else L.W97
    h, w = coef.shape[-2:]
    odt = torch.int32 if kernel == L.W53 else torch.float32
    if out is None:
        out = torch.empty(coef.shape, dtype=odt, device=coef.device)
    keep, sp = _steps_arg(steps, levels)
    hh = ctx._bind()
    if coef.dim() == 3:
        check(lib().j2k_dwt_inverse_batch(hh, kernel, order, _ptr(coef), coef.stride(1), coef.stride(0),
                                          _ptr(out), out.stride(1), out.stride(0), coef.shape[0], w, h,
                                          levels, sp), hh)
    else:
        check(lib().j2k_dwt_inverse(hh, kernel, order, _ptr(coef), coef.stride(0), _ptr(out),
                                    out.stride(0), w, h, levels, sp), hh)
    return out


def codeblock_count(w, h, levels, cbw=64, cbh=64):
    return int(lib().j2k_codeblock_count(w, h, levels, cbw, cbh))


def bpc_encode(coef, levels, cbw=64, cbh=64, cap_per_block=None, ctx=None):
    """Tier-1 encode of every code-block of an int32 Mallat plane.
    Returns (descs: numpy structured array, bytes: uint8 CUDA tensor of count*cap)."""
    ctx = ctx or default_context(coef.device.index or 0)
    _need_cuda(coef, "coef")
    h, w = coef.shape
    n = codeblock_count(w, h, levels, cbw, cbh)
    cap = cap_per_block or ((cbw * cbh * 2 + 256 + 15) // 16 * 16)
    descs = torch.empty(n * 24, dtype=torch.uint8, device=coef.device)
    out = torch.empty(n * cap, dtype=torch.uint8, device=coef.device)
    hh = ctx._bind()
    check(lib().j2k_bpc_encode(hh, _ptr(coef), coef.stride(0), w, h, levels, cbw, cbh, _ptr(descs),
                               _ptr(out), cap), hh)
    return descs.cpu().numpy().view(L.CB_DESC), out


def bpc_decode(descs, data, w, h, levels, cbw=64, cbh=64, ctx=None, out=None):
    """descs: numpy structured array (host) or uint8 CUDA tensor; data: uint8 CUDA tensor."""
    ctx = ctx or default_context(data.device.index or 0)
    _need_cuda(data, "data")
    if isinstance(descs, np.ndarray):
        d = torch.from_numpy(np.ascontiguousarray(descs).view(np.uint8)).to(data.device)
        n = descs.shape[0]
    else:
        d, n = descs, descs.numel() // 24
    if out is None:
        out = torch.empty((h, w), dtype=torch.int32, device=data.device)
    hh = ctx._bind()
    check(lib().j2k_bpc_decode(hh, _ptr(d), _ptr(data), n, _ptr(out), out.stride(0), w, h, levels,
                               cbw, cbh), hh)
    return out


# ---------------------------------------------------------------------------------------------
# Reference-shaped classes
# ---------------------------------------------------------------------------------------------

def _params(levels, cbw, cbh, order, steps, target_bytes=0, layers=None, cblk_style=0, pass_ends=None):
    keep, sp = _steps_arg(steps, levels) if steps is not None else (None, None)
    nl, lp = 0, None
    if layers is not None and len(layers) > 1:
        lb = np.ascontiguousarray(np.asarray(layers, np.uint64))
        keep = (keep, lb)
        nl, lp = len(lb), lb.ctypes.data
    pe = None
    if pass_ends is not None:
        pea = np.ascontiguousarray(pass_ends, np.uint32)
        keep = (keep, pea)
        pe = pea.ctypes.data
    p = L.EncParams(levels, cbw, cbh, order, sp, int(target_bytes), nl, lp, int(cblk_style), pe)
    return p, keep


class OCLEncodeDecode:
    """Common base (src/OCLEncodeDecode.h:23-38): owns the device context."""

    def __init__(self, ctx=None, lossy=False, output_dwt=False):
        self.ctx = ctx or default_context(0)
        self.lossy = bool(lossy)
        self.output_dwt = bool(output_dwt)

    def finish(self):
        """clFinish equivalent (src/OCLEncodeDecode.cpp:33-36)."""
        self.ctx.sync()


class OCLEncoder(OCLEncodeDecode):
    """OCLEncoder<T> (src/OCLEncoder.cpp:26-52)."""

    def __init__(self, ctx=None, lossy=False, output_dwt=False):
        super().__init__(ctx, lossy, output_dwt)
        h = C.c_void_p()
        check(lib().j2k_encoder_create(self.ctx.h, int(self.lossy), int(self.output_dwt), C.byref(h)),
              self.ctx.h)
        self.h = h
        self.w = self.h_ = self.ncomp = self.levels = 0

    def __del__(self):
        try:
            if self.h:
                lib().j2k_encoder_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def run(self, components, w, h, levels, precision=8, cbw=64, cbh=64, order=L.ORDER_T800,
            steps=None, target_bytes=0, layers=None):
        """Reference signature: planar host components (numpy int16/int32/float32, already
        level-shifted by -128, as src/OCLTest.cpp:80-90 builds them).  target_bytes > 0 cuts the
        codestream to at most that many bytes (PCRD-opt rate control); layers = cumulative byte
        budgets of several quality layers (see run_rgb)."""
        comps = [np.ascontiguousarray(c) for c in components]
        dt = {np.dtype(np.int16): L.I16, np.dtype(np.int32): L.I32, np.dtype(np.float32): L.F32}[comps[0].dtype]
        arr = (C.c_void_p * len(comps))(*[c.ctypes.data for c in comps])
        p, keep = _params(levels, cbw, cbh, order, steps, target_bytes, layers)
        hh = self.ctx._bind()
        check(lib().j2k_encoder_run(self.h, arr, len(comps), dt, w, h, levels, precision, C.byref(p)), hh)
        self.w, self.h_, self.ncomp, self.levels = w, h, len(comps), levels
        return self

    def autotune(self, reps=2):
        """Times the tier-1 MQ warp schedules on the last run's coefficients and keeps the fastest
        in this encoder's context (shared with every object on that context)."""
        rep = (C.c_int * 4)()
        hh = self.ctx._bind()
        check(lib().j2k_encoder_autotune(self.h, reps, rep), hh)
        return {"tier0_warps": rep[0], "tier1_warps": rep[1], "tier1_blocks_per_warp": rep[2],
                "blocks_per_warp": rep[3]}

    def run_rgb(self, img, levels=5, cbw=64, cbh=64, order=L.ORDER_T800, steps=None, target_bytes=0,
                layers=None, cblk_style=0):
        """Interleaved uint8 image, (H, W, C) or (H, W); numpy (host) or CUDA tensor.
        target_bytes > 0 cuts the codestream to at most that many bytes (PCRD-opt rate control:
        bit-plane truncation points of every code-block chosen on their rate-distortion hulls).
        layers: cumulative codestream byte budgets of quality layers 0, 1, ... (non-decreasing;
        a last entry of 0 keeps every pass, a lossless final layer for 5/3).  cblk_style:
        code-block style bits (CBLK_BYPASS | CBLK_RESET | CBLK_TERMALL; not with rate control);
        with RESET and TERMALL the passes of a block are coded in parallel."""
        if isinstance(img, torch.Tensor) and img.is_cuda:
            t = img.contiguous()
            ptr, on_dev = t.data_ptr(), 1
            hgt, wid = t.shape[0], t.shape[1]
            nc = 1 if t.dim() == 2 else t.shape[2]
            keep_img = t
        else:
            a = np.ascontiguousarray(img if not isinstance(img, torch.Tensor) else img.numpy(), np.uint8)
            ptr, on_dev = a.ctypes.data, 0
            hgt, wid = a.shape[0], a.shape[1]
            nc = 1 if a.ndim == 2 else a.shape[2]
            keep_img = a
        p, keep = _params(levels, cbw, cbh, order, steps, target_bytes, layers, cblk_style)
        hh = self.ctx._bind()
        check(lib().j2k_encoder_run_interleaved(self.h, C.c_void_p(ptr), on_dev, wid * nc, nc, wid, hgt,
                                                C.byref(p)), hh)
        del keep_img
        self.w, self.h_, self.ncomp, self.levels = wid, hgt, nc, levels
        self.cblk_style = int(cblk_style)
        return self

    def get_pass_ends(self):
        """Pass ends of the last styled run: (count, PASS_STRIDE) uint32, row i for code-block i
        (job order), entry p the codeword bytes when pass p ended (exact where the style
        terminates the codeword after it)."""
        n = C.c_size_t()
        check(lib().j2k_encoder_get_pass_ends(self.h, None, 0, C.byref(n)), self.ctx.h)
        out = np.zeros(n.value, np.uint32)
        check(lib().j2k_encoder_get_pass_ends(self.h, out.ctypes.data_as(C.c_void_p), out.size, C.byref(n)),
              self.ctx.h)
        return out.reshape(-1, L.PASS_STRIDE)

    def map_dwt_out(self):
        """Host copy of the coefficient planes: (ncomp, H, W) int32 (float32 for lossy DWT-only)."""
        ptr, pitch = C.c_void_p(), C.c_size_t()
        check(lib().j2k_encoder_map_dwt_out(self.h, C.byref(ptr), C.byref(pitch)), self.ctx.h)
        dt = np.float32 if (self.lossy and self.output_dwt) else np.int32
        n = self.ncomp * self.h_ * self.w
        buf = (C.c_char * (n * 4)).from_address(ptr.value)
        out = np.frombuffer(buf, dtype=dt, count=n).reshape(self.ncomp, self.h_, self.w).copy()
        check(lib().j2k_encoder_unmap_dwt_out(self.h, ptr), self.ctx.h)
        return out

    def get_codeblocks(self, pinned=False):
        """(descs structured array, packed codeword bytes) copied to the host.  With pinned=True
        the copies land in page-locked buffers owned by the encoder (a faster transfer) and the
        returned arrays are views of them, valid until the next get_codeblocks call."""
        cnt, used = C.c_size_t(), C.c_size_t()
        check(lib().j2k_encoder_get_codeblocks(self.h, None, C.byref(cnt), None, 0, C.byref(used)),
              self.ctx.h)
        nd, nb = cnt.value * L.CB_DESC.itemsize, max(used.value, 1)
        if pinned:
            pd, pb = getattr(self, "_pin_d", None), getattr(self, "_pin_b", None)
            if pd is None or pd.numel() < nd:
                self._pin_d = pd = torch.empty(nd, dtype=torch.uint8, pin_memory=True)
            if pb is None or pb.numel() < nb:
                self._pin_b = pb = torch.empty(nb + nb // 4, dtype=torch.uint8, pin_memory=True)
            d = pd.numpy()[:nd].view(L.CB_DESC)
            b = pb.numpy()
        else:
            d = np.zeros(cnt.value, L.CB_DESC)
            b = np.zeros(nb, np.uint8)
        check(lib().j2k_encoder_get_codeblocks(self.h, d.ctypes.data_as(C.c_void_p), C.byref(cnt),
                                               b.ctypes.data_as(C.c_void_p), b.size, C.byref(used)),
              self.ctx.h)
        return d, b[:used.value]

    def codestream(self):
        n = C.c_size_t()
        check(lib().j2k_encoder_get_codestream(self.h, None, 0, C.byref(n)), self.ctx.h)
        out = np.zeros(n.value, np.uint8)
        check(lib().j2k_encoder_get_codestream(self.h, out.ctypes.data_as(C.c_void_p), out.size,
                                               C.byref(n)), self.ctx.h)
        return out.tobytes()

    def device_results(self):
        d, b, cnt, cap = C.c_void_p(), C.c_void_p(), C.c_size_t(), C.c_size_t()
        check(lib().j2k_encoder_device_results(self.h, C.byref(d), C.byref(b), C.byref(cnt), C.byref(cap)),
              self.ctx.h)
        return d.value, b.value, cnt.value, cap.value


class OCLDecoder(OCLEncodeDecode):
    """OCLDecoder<T> (src/OCLDecoder.cpp:24-38), decoding code-blocks back to pixels."""

    def __init__(self, ctx=None, lossy=False):
        super().__init__(ctx, lossy, False)
        h = C.c_void_p()
        check(lib().j2k_decoder_create(self.ctx.h, int(self.lossy), C.byref(h)), self.ctx.h)
        self.h = h

    def __del__(self):
        try:
            if self.h:
                lib().j2k_decoder_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def run(self, descs, data, w, h, ncomp, levels=5, cbw=64, cbh=64, order=L.ORDER_T800, steps=None,
            cblk_style=0, pass_ends=None, out=None):
        """descs/data as returned by OCLEncoder.get_codeblocks (host).  Returns (H, W, C) uint8:
        `out` when given (a C-contiguous (H, W, C) uint8 host array, e.g. page-locked memory,
        which the pixels are copied into directly), else a new array.  Blocks coded with a
        code-block style need cblk_style and their pass ends (OCLEncoder.get_pass_ends,
        read_pass_ends)."""
        descs = np.ascontiguousarray(descs)
        data = np.ascontiguousarray(data, np.uint8)
        if out is None:
            out = np.zeros((h, w, ncomp), np.uint8)
        elif (out.dtype != np.uint8 or out.shape != (h, w, ncomp) or not out.flags["C_CONTIGUOUS"]
              or not out.flags["WRITEABLE"]):
            raise ValueError(f"out must be a writeable C-contiguous uint8 array of shape {(h, w, ncomp)}")
        if cblk_style and pass_ends is None:
            raise ValueError("a styled decode needs the pass ends")
        p, keep = _params(levels, cbw, cbh, order, steps, cblk_style=cblk_style, pass_ends=pass_ends)
        hh = self.ctx._bind()
        check(lib().j2k_decoder_run_codeblocks(self.h, descs.ctypes.data_as(C.c_void_p),
                                               data.ctypes.data_as(C.c_void_p), data.size, 0, ncomp,
                                               w, h, C.byref(p), out.ctypes.data_as(C.c_void_p), 0,
                                               w * ncomp), hh)
        return out


def read_codestream(cs, max_layers=0):
    """Tier-2 decoding of a codestream (bytes): -> (info dict, descs structured array, codeword
    bytes), ready for OCLDecoder.run.  Every quality layer is parsed; a block's codeword is the
    concatenation of its segments from the first `max_layers` layers (0: all), so a prefix of the
    layers decodes to the image at that quality.  Raises J2KError(J2K_ERR_UNSUPPORTED) with the
    reason for streams outside the supported subset (one tile, LRCP/RLCP, default code-block
    style, 1 or 3 colour-transformed 8-bit components)."""
    buf = np.frombuffer(bytes(cs), np.uint8)
    info = L.StreamInfo()
    cnt, used = C.c_size_t(), C.c_size_t()
    err = C.create_string_buffer(256)
    s = lib().j2k_codestream_read_layers(buf.ctypes.data_as(C.c_void_p), buf.size, int(max_layers), C.byref(info),
                                         None, C.byref(cnt), None, 0, C.byref(used), err, 256)
    if s != 0:
        raise L.J2KError(s, err.value.decode())
    descs = np.zeros(cnt.value, L.CB_DESC)
    data = np.zeros(max(used.value, 1), np.uint8)
    s = lib().j2k_codestream_read_layers(buf.ctypes.data_as(C.c_void_p), buf.size, int(max_layers), C.byref(info),
                                         descs.ctypes.data_as(C.c_void_p), C.byref(cnt),
                                         data.ctypes.data_as(C.c_void_p), data.size, C.byref(used), err, 256)
    if s != 0:
        raise L.J2KError(s, err.value.decode())
    nb = 3 * info.levels + 1
    d = dict(w=info.w, h=info.h, ncomp=info.ncomp, levels=info.levels, cbw=info.cbw, cbh=info.cbh,
             lossless=bool(info.lossless), mct=info.mct, guard=info.guard, precision=info.precision,
             layers=info.layers, progression=info.progression, cblk_style=info.cblk_style,
             steps=np.array(info.steps[:nb], np.float32))
    return d, descs, data[:used.value]


def read_pass_ends(cs, max_layers=0):
    """Pass ends of the blocks read_codestream returns: (count, PASS_STRIDE) uint32 (for a
    styled stream's decode; an unstyled stream gives each block's codeword length)."""
    buf = np.frombuffer(bytes(cs), np.uint8)
    n = C.c_size_t()
    err = C.create_string_buffer(256)
    s = lib().j2k_codestream_pass_ends(buf.ctypes.data_as(C.c_void_p), buf.size, int(max_layers), None, 0,
                                       C.byref(n), err, 256)
    if s != 0:
        raise L.J2KError(s, err.value.decode())
    out = np.zeros(n.value, np.uint32)
    s = lib().j2k_codestream_pass_ends(buf.ctypes.data_as(C.c_void_p), buf.size, int(max_layers),
                                       out.ctypes.data_as(C.c_void_p), out.size, C.byref(n), err, 256)
    if s != 0:
        raise L.J2KError(s, err.value.decode())
    return out.reshape(-1, L.PASS_STRIDE)


def write_codestream(w, h, ncomp, levels, descs, data, cbw=64, cbh=64, lossless=True, steps=None, layers=None):
    """Tier-2 only (host): the codestream of code-blocks coded elsewhere.  descs/data as
    get_codeblocks or read_codestream return them (job order).  layers: None for one layer, or
    (npasses, lengths), two (L, count) int arrays of what each block holds after each layer."""
    descs = np.ascontiguousarray(descs)
    data = np.ascontiguousarray(data, np.uint8)
    st = None if steps is None else np.ascontiguousarray(steps, np.float32)
    nl, lp, ll = 0, None, None
    if layers is not None:
        lp = np.ascontiguousarray(layers[0], np.int32)
        ll = np.ascontiguousarray(layers[1], np.int32)
        if lp.shape != ll.shape or lp.ndim != 2 or lp.shape[1] != descs.size:
            raise ValueError("layers: two (L, count) arrays")
        nl = lp.shape[0]
    args = (w, h, ncomp, levels, cbw, cbh, int(lossless), None if st is None else st.ctypes.data,
            descs.ctypes.data, descs.size, data.ctypes.data, data.size, nl,
            None if lp is None else lp.ctypes.data, None if ll is None else ll.ctypes.data)
    n = C.c_size_t()
    s = lib().j2k_codestream_write(*args, None, 0, C.byref(n))
    if s != 0:
        raise L.J2KError(s, "j2k_codestream_write: invalid arguments")
    out = np.zeros(n.value, np.uint8)
    s = lib().j2k_codestream_write(*args, out.ctypes.data, out.size, C.byref(n))
    if s != 0:
        raise L.J2KError(s, "j2k_codestream_write failed")
    return out.tobytes()


def decode_codestream(cs, ctx=None, max_layers=0):
    """Decodes a codestream on the GPU: tier-2 on the host, then tier-1, inverse DWT and inverse
    colour transform on the device.  max_layers > 0 decodes only the first quality layers.
    Returns (H, W, C) uint8."""
    info, descs, data = read_codestream(cs, max_layers)
    pe = read_pass_ends(cs, max_layers) if info["cblk_style"] else None
    dec = OCLDecoder(ctx=ctx, lossy=not info["lossless"])
    return dec.run(descs, data, info["w"], info["h"], info["ncomp"], levels=info["levels"], cbw=info["cbw"],
                   cbh=info["cbh"], steps=None if info["lossless"] else info["steps"],
                   cblk_style=info["cblk_style"], pass_ends=pe)


def codestream_info(cs):
    """The main header of a codestream (no packet is parsed): w, h, ncomp, levels, ..."""
    buf = np.frombuffer(bytes(cs), np.uint8)
    info = L.StreamInfo()
    err = C.create_string_buffer(256)
    s = lib().j2k_codestream_info(buf.ctypes.data_as(C.c_void_p), buf.size, C.byref(info), err, 256)
    if s != 0:
        raise L.J2KError(s, err.value.decode())
    return dict(w=info.w, h=info.h, ncomp=info.ncomp, levels=info.levels, cbw=info.cbw, cbh=info.cbh,
                lossless=bool(info.lossless), layers=info.layers, progression=info.progression)


def decode_codestreams(streams, ctx=None, max_layers=0, decoder=None):
    """Batched GPU decode of many codestreams: tier-2 of every stream on a pool of host threads,
    then one upload of all code-blocks, one tier-1 launch over every block of every image, the
    inverse DWT and colour transform per image, and one read-back.  Returns a list of
    (H, W[, C]) uint8 arrays."""
    ctx = ctx or default_context(0)
    bufs = [np.frombuffer(bytes(cs), np.uint8) for cs in streams]
    outs = []
    for b in bufs:
        info = codestream_info(b)
        nc = info["ncomp"]
        outs.append(np.empty((info["h"], info["w"], nc) if nc > 1 else (info["h"], info["w"]), np.uint8))
    n = len(bufs)
    sp = (C.c_void_p * n)(*[b.ctypes.data for b in bufs])
    sz = (C.c_size_t * n)(*[b.size for b in bufs])
    op = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
    dec = decoder or OCLDecoder(ctx=ctx)  # a kept decoder reuses its device buffers
    hh = dec.ctx._bind()
    check(lib().j2k_decoder_run_codestreams(dec.h, sp, sz, n, int(max_layers), op), hh)
    return outs


class OCLDWTForward:
    """OCLDWTForward<T>::run(lossy, w, h, windowX, windowY, level, levels) (src/OCLDWTForward.h:31).
    The window arguments of the OpenCL launch geometry have no meaning here and are ignored."""

    def __init__(self, ctx=None, order=L.ORDER_REF):
        self.ctx = ctx or default_context(0)
        self.order = order

    def run(self, plane, lossy, w=None, h=None, windowX=None, windowY=None, level=0, levels=1,
            steps=None):
        return dwt_forward(plane, levels - level, L.W97 if lossy else L.W53, self.order, steps, self.ctx)


class OCLDWTRev:
    """OCLDWTRev<T>::run(lossy, w, h, windowX, windowY) (src/OCLDWTRev.h:31) as a true inverse."""

    def __init__(self, ctx=None, order=L.ORDER_REF):
        self.ctx = ctx or default_context(0)
        self.order = order

    def run(self, coef, lossy, w=None, h=None, windowX=None, windowY=None, levels=1, steps=None):
        return dwt_inverse(coef, levels, L.W97 if lossy else L.W53, self.order, steps, self.ctx)


class OCLRGBtoPlanar:
    """OCLRGBtoPlanar<T>::run() (src/OCLRGBtoPlanar.h:28), with the colour transform fused."""

    def __init__(self, ctx=None, mct=L.MCT_RCT):
        self.ctx = ctx or default_context(0)
        self.mct = mct

    def run(self, img):
        return rgb_to_planar(img, self.mct, self.ctx)


class OCLBPC:
    """OCLBPC<T>::run(codeblockX, codeblockY) (src/OCLBPC.h:28), producing real codewords."""

    def __init__(self, ctx=None):
        self.ctx = ctx or default_context(0)

    def run(self, coef, levels, codeblockX=64, codeblockY=64):
        return bpc_encode(coef, levels, codeblockX, codeblockY, ctx=self.ctx)
