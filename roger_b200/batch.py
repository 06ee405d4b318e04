"""Batched encoder over the C ABI (j2k_batch_*): many images of uneven size, mixed 5/3 and 9/7,
encoded by one fixed launch sequence (replayed as a CUDA graph).  No reference counterpart:
the reference encodes one image per OCLEncoder<T>::run call (src/OCLEncoder.cpp:43-52)."""
import ctypes as C

import numpy as np
import torch

from . import _lib as L
from ._lib import check, lib

TILE_NAMES = {0: "64x64", 1: "128x32", 2: "32x128", 3: "248x16 register lifting"}


def split_packed(first, descs, data):
    """Per-image (descs, codeword bytes) of a packed batch result: image i owns descriptors
    first[i]:first[i+1], whose offsets point into `data` back to back in job order.  The
    descriptors come back as one rebased copy (offsets relative to each image's bytes) and the
    bytes as views of `data`."""
    first = np.asarray(first, np.int64)
    n = len(first) - 1
    d = np.ascontiguousarray(descs[:first[-1]]).view(np.uint8).copy().view(descs.dtype)  # a byte copy
    counts = np.diff(first)
    has = counts > 0
    base = np.zeros(n, np.int64)
    base[has] = d["offset"][first[:-1][has]]
    end = base.copy()
    last = first[1:][has] - 1
    end[has] = d["offset"][last].astype(np.int64) + np.maximum(d["length"][last], 0)
    d["offset"] -= np.repeat(base, counts).astype(d["offset"].dtype)
    return [(d[first[i]:first[i + 1]], data[base[i]:end[i]]) for i in range(n)]


class BatchEncoder:
    """images: list of dicts with w, h, ncomp (1|3), kernel (53|97), levels, cb[, steps]."""

    def __init__(self, images, ctx=None):
        # a context of its own by default: autotune() sets the context's tier-1 schedule
        from .codec import Context
        self.ctx = ctx or Context(0)
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

    def encode(self, images=None, wait=True):
        """Encodes the batch; images=None re-encodes what is already in the input buffer.
        wait=False queues the work on the current stream and returns at once (the device error
        word is read by the next call that needs the result); host images must then stay alive
        until the stream has copied them."""
        hh = self.ctx._bind()
        fn = lib().j2k_batch_encode if wait else lib().j2k_batch_encode_async
        if images is None:
            check(fn(self.h, None, 0), hh)
        else:
            ptrs, on_dev, keep = self.load(images)
            self._keep = keep
            check(fn(self.h, ptrs, on_dev), hh)
        return self

    def upload(self, images):
        """Queues only the copies of the images into the input buffer on the current stream."""
        hh = self.ctx._bind()
        ptrs, on_dev, keep = self.load(images)
        self._keep = keep
        check(lib().j2k_batch_upload(self.h, ptrs, on_dev), hh)
        return self

    def set_option(self, key, value):
        check(lib().j2k_batch_set_option(self.h, key, value), self.ctx.h)

    def get_option(self, key):
        v = C.c_int()
        check(lib().j2k_batch_get_option(self.h, key, C.byref(v)), self.ctx.h)
        return v.value

    def autotune(self, reps=2):
        rep = (C.c_int * 5)()
        hh = self.ctx._bind()
        check(lib().j2k_batch_autotune(self.h, reps, rep), hh)
        tiers = C.c_int()
        check(lib().j2k_batch_get_option(self.h, 7, C.byref(tiers)), hh)
        mq = "state+code warp pair" if rep[3] else f"one lane per block, {rep[4]} per warp"
        if tiers.value and not rep[3]:
            mq += " after the tiers (longest blocks: 1 per warp, then 4 per warp)"
        return {"tile53": TILE_NAMES[rep[0]], "tile97": TILE_NAMES[rep[1]],
                "phase_a_order": "largest-first" if rep[2] else "natural", "mq": mq,
                "phase_a_ctas_per_sm": self.get_option(10)}

    def results(self, pinned=True):
        """Every image's (descs, codeword bytes), read back in one packing pass and two copies
        (into reused page-locked buffers when pinned; views valid until the next call)."""
        self.read_async(pinned)
        torch.cuda.current_stream().synchronize()
        return self.split()

    def read_async(self, pinned=True):
        """Packs the results on the device and queues their copy to the host on the current
        stream without waiting (split() after the stream has finished gives the per-image
        views).  Waits only for the packed size."""
        hh = self.ctx._bind()
        total = C.c_size_t()
        check(lib().j2k_batch_pack(self.h, C.byref(total)), hh)
        first = (C.c_size_t * (len(self.desc) + 1))()
        check(lib().j2k_batch_image_jobs(self.h, first), hh)
        self._first = [first[i] for i in range(len(self.desc) + 1)]
        nd, nb = self._first[-1] * L.CB_DESC.itemsize, max(total.value, 1)
        if pinned:
            pd, pb = getattr(self, "_pin_d", None), getattr(self, "_pin_b", None)
            if pd is None or pd.numel() < nd:
                self._pin_d = pd = torch.empty(nd, dtype=torch.uint8, pin_memory=True)
            if pb is None or pb.numel() < nb:
                self._pin_b = pb = torch.empty(nb + nb // 4, dtype=torch.uint8, pin_memory=True)
            self._d = pd.numpy()[:nd].view(L.CB_DESC)
            self._b = pb.numpy()
        else:
            self._d = np.zeros(self._first[-1], L.CB_DESC)
            self._b = np.zeros(nb, np.uint8)
        self._total = total.value
        check(lib().j2k_batch_read_packed(self.h, self._d.ctypes.data_as(C.c_void_p),
                                          self._b.ctypes.data_as(C.c_void_p), self._b.size), hh)

    def split(self):
        return split_packed(self._first, self._d, self._b)

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


class StreamingBatchEncoder:
    """Encodes a stream of batches of one layout (same image shapes and settings) from host
    memory to host memory, with the copies overlapped: while batch k is encoded (one batched
    graph on the compute stream), batch k+1's pixels go up on a copy stream and batch k-1's
    packed code-blocks come back on their own stream.  `depth` batched encoders (each with its
    own context and device buffers) take turns; in steady state a batch costs the larger of its
    encode and its copies instead of their sum.  Splitting one batch into groups that take
    turns does not pay: tier-1 time is set by the longest code-blocks of each launch, so every
    extra launch adds its own tail.

    Host images should be page-locked (`pin`) for the copies to be asynchronous.  The results
    of a batch are views into page-locked buffers of its encoder, valid until that encoder's
    turn comes again (`depth` batches later)."""

    def __init__(self, images, depth=2, device=0):
        from .codec import Context
        self.desc = list(images)
        self.depth = max(2, depth)
        self.encs = [BatchEncoder(self.desc, ctx=Context(device)) for _ in range(self.depth)]
        self.compute = torch.cuda.Stream(device=device)
        self.copy = torch.cuda.Stream(device=device)
        self.out = [torch.cuda.Stream(device=device) for _ in range(self.depth)]
        self.computed = [None] * self.depth

    @staticmethod
    def pin(images):
        """Page-locked host copies of numpy images (made once, outside any timed region)."""
        return [torch.from_numpy(np.ascontiguousarray(im)).pin_memory().numpy() for im in images]

    def autotune(self, images, reps=1):
        for e in self.encs:
            e.encode(images)
            e.autotune(reps=reps)

    def _start(self, k, images):
        i = k % self.depth
        enc = self.encs[i]
        if self.computed[i] is not None:  # the input buffer is free once its last encode ran
            self.copy.wait_event(self.computed[i])
        with torch.cuda.stream(self.copy):
            enc.upload(images)
            up = torch.cuda.Event()
            up.record(self.copy)
        self.compute.wait_event(up)
        with torch.cuda.stream(self.compute):
            enc.encode(None, wait=False)
            ev = torch.cuda.Event()
            ev.record(self.compute)
        self.computed[i] = ev

    def _finish(self, k):
        i = k % self.depth
        s = self.out[i]
        s.wait_event(self.computed[i])
        with torch.cuda.stream(s):
            self.encs[i].read_async(pinned=True)
        s.synchronize()
        return self.encs[i].split()

    def run(self, batches):
        """batches: iterable of lists of host images (batch order).  Yields, per batch in order,
        every image's (descs, codeword bytes)."""
        k = -1
        for k, images in enumerate(batches):
            self._start(k, images)
            if k >= 1:
                yield self._finish(k - 1)
        if k >= 0:
            yield self._finish(k)
