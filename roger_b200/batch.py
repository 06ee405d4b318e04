"""Batched encoder over the C ABI (j2k_batch_*): many images of uneven size, mixed 5/3 and 9/7,
encoded by one fixed launch sequence (replayed as a CUDA graph).  No reference counterpart:
the reference encodes one image per OCLEncoder<T>::run call (src/OCLEncoder.cpp:43-52)."""
import ctypes as C

import numpy as np
import torch

from . import _lib as L
from ._lib import check, lib
from .codec import default_context

TILE_NAMES = {0: "64x64", 1: "128x32", 2: "32x128"}


class BatchEncoder:
    """images: list of dicts with w, h, ncomp (1|3), kernel (53|97), levels, cb[, steps]."""

    def __init__(self, images, ctx=None):
        self.ctx = ctx or default_context(0)
        self.desc = list(images)
        n = len(self.desc)
        arr = (L.BatchImage * n)()
        self._steps = []
        for i, d in enumerate(self.desc):
            st = None
            if d.get("steps") is not None:
                a = np.ascontiguousarray(d["steps"], np.float32)
                self._steps.append(a)
                st = a.ctypes.data
            arr[i] = L.BatchImage(d["w"], d["h"], d["ncomp"], d["kernel"], d["levels"], d["cb"], st)
        h = C.c_void_p()
        check(lib().j2k_batch_create(self.ctx.h, arr, n, C.byref(h)), self.ctx.h)
        self.h = h
        buf = C.c_void_p()
        offs = (C.c_size_t * (n + 1))()
        check(lib().j2k_batch_input(self.h, C.byref(buf), offs), self.ctx.h)
        self.input_ptr = buf.value
        self.offsets = [offs[i] for i in range(n + 1)]

    def __del__(self):
        try:
            if self.h:
                lib().j2k_batch_destroy(self.h)
                self.h = None
        except Exception:
            pass

    @property
    def pixels(self):
        return sum(d["w"] * d["h"] for d in self.desc)

    def load(self, images):
        """Copies images (numpy or CUDA tensors, (h, w[, c]) uint8) into the device input buffer."""
        ptrs = (C.c_void_p * len(images))()
        keep = []
        on_dev = None
        for i, im in enumerate(images):
            if isinstance(im, torch.Tensor) and im.is_cuda:
                t = im.contiguous()
                keep.append(t)
                ptrs[i] = t.data_ptr()
                dev = 1
            else:
                a = np.ascontiguousarray(im.numpy() if isinstance(im, torch.Tensor) else im, np.uint8)
                keep.append(a)
                ptrs[i] = a.ctypes.data
                dev = 0
            if on_dev is None:
                on_dev = dev
            elif on_dev != dev:
                raise ValueError("images must be all on the host or all on the device")
        return ptrs, on_dev, keep

    def encode(self, images=None):
        """Encodes the batch; images=None re-encodes what is already in the input buffer."""
        hh = self.ctx._bind()
        if images is None:
            check(lib().j2k_batch_encode(self.h, None, 0), hh)
        else:
            ptrs, on_dev, keep = self.load(images)
            check(lib().j2k_batch_encode(self.h, ptrs, on_dev), hh)
        return self

    def set_option(self, key, value):
        check(lib().j2k_batch_set_option(self.h, key, value), self.ctx.h)

    def autotune(self, reps=2):
        rep = (C.c_int * 5)()
        hh = self.ctx._bind()
        check(lib().j2k_batch_autotune(self.h, reps, rep), hh)
        return {"tile53": TILE_NAMES[rep[0]], "tile97": TILE_NAMES[rep[1]],
                "phase_a_order": "largest-first" if rep[2] else "natural",
                "mq": ("state+code warp pair" if rep[3] else f"one lane per block, {rep[4]} per warp")}

    def codeblocks(self, i):
        cnt, used = C.c_size_t(), C.c_size_t()
        check(lib().j2k_batch_get_codeblocks(self.h, i, None, C.byref(cnt), None, 0, C.byref(used)), self.ctx.h)
        d = np.zeros(cnt.value, L.CB_DESC)
        b = np.zeros(max(used.value, 1), np.uint8)
        check(lib().j2k_batch_get_codeblocks(self.h, i, d.ctypes.data_as(C.c_void_p), C.byref(cnt),
                                             b.ctypes.data_as(C.c_void_p), b.size, C.byref(used)), self.ctx.h)
        return d, b[:used.value]

    def codestream(self, i):
        n = C.c_size_t()
        check(lib().j2k_batch_get_codestream(self.h, i, None, 0, C.byref(n)), self.ctx.h)
        out = np.zeros(n.value, np.uint8)
        check(lib().j2k_batch_get_codestream(self.h, i, out.ctypes.data_as(C.c_void_p), out.size, C.byref(n)),
              self.ctx.h)
        return out.tobytes()
