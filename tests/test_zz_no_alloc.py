"""GPU test of the allocation-free forward DWT (j2k_dwt_forward_noalloc), called through the C
ABI.  It serves callers that cannot allocate device memory (a plugin inside a framework that
owns the device heap, a pipeline that must never reach cudaMalloc); its output must equal the
regular j2k_dwt_forward's on two calls in a row, since the calls share one reserved array.

This file is collected last on purpose, so that a run stopping at the first failure has run
every other test first.  The first call on a device looks up the reserved array's address;
test_noalloc_first_call_in_a_fresh_process covers that first call in a process of its own."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
REL_TOL_97 = 1e-4
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _noalloc(x, out, kernel, order, levels, steps=None, w=None, h=None):
    from roger_b200 import _lib
    st = None
    keep = None
    if steps is not None:
        keep = np.ascontiguousarray(steps, np.float32)
        st = keep.ctypes.data_as(C.c_void_p)
    hh, ww = x.shape
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return _lib.lib().j2k_dwt_forward_noalloc(stream, kernel, order, C.c_void_p(x.data_ptr()), x.stride(0),
                                             C.c_void_p(out.data_ptr()), out.stride(0), w or ww, h or hh,
                                             levels, st)


@pytest.mark.parametrize("kernel,w,h,levels,order,quant", [
    (53, 2048, 2048, 6, 0, False), (53, 1001, 777, 5, 1, False), (97, 1024, 768, 5, 0, False),
    (97, 2048, 2048, 6, 0, True), (53, 3, 5, 2, 0, False)])
def test_noalloc_matches_regular_dwt_twice(kernel, w, h, levels, order, quant):
    from roger_b200 import codec
    rng = np.random.default_rng(w * 31 + h)
    if kernel == 53:
        x = torch.from_numpy(rng.integers(-255, 256, (h, w)).astype(np.int32)).cuda()
    else:
        x = torch.from_numpy(rng.uniform(-128, 128, (h, w)).astype(np.float32)).cuda()
    steps = codec.default_steps(w, h, levels) if quant else None
    ref = codec.dwt_forward(x, levels, kernel, order, steps=steps).cpu().numpy()
    odt = torch.int32 if (kernel == 53 or quant) else torch.float32
    for _ in range(2):
        out = torch.full((h, w), 7, dtype=odt, device="cuda")
        assert _noalloc(x, out, kernel, order, levels, steps) == 0
        got = out.cpu().numpy()
        if odt == torch.float32:
            peak = max(float(np.abs(ref).max()), 1e-6)
            assert float(np.abs(got - ref).max()) / peak <= REL_TOL_97
        else:
            assert np.array_equal(got, ref)


def test_noalloc_rejects_images_beyond_its_reserved_array():
    x = torch.zeros((2049, 2048), dtype=torch.int32, device="cuda")
    out = torch.zeros_like(x)
    assert _noalloc(x, out, 53, 0, 3) == -5   # J2K_ERR_CAPACITY, nothing launched
    # sizes beyond 31 bits are refused before any size arithmetic (J2K_ERR_INVALID_ARG); the
    # pitch passes, so the check itself is what refuses them, and nothing is launched
    y = torch.zeros((1, 8), dtype=torch.int32, device="cuda")
    big = 1 << 31
    from roger_b200 import _lib
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for w, h in [(big, 1), (1, big), (big + 3, big + 3)]:
        r = _lib.lib().j2k_dwt_forward_noalloc(stream, 53, 0, C.c_void_p(y.data_ptr()), big + 8,
                                              C.c_void_p(y.data_ptr()), big + 8, w, h, 1, None)
        assert r == -1


_FRESH = r"""
import ctypes as C, sys
import numpy as np, torch
sys.path.insert(0, {root!r})
from roger_b200 import _lib, codec
rng = np.random.default_rng(5)
x = torch.from_numpy(rng.integers(-255, 256, (600, 700)).astype(np.int32)).cuda()
out = torch.full_like(x, 7)
s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
for _ in range(2):
    r = _lib.lib().j2k_dwt_forward_noalloc(s, 53, 0, C.c_void_p(x.data_ptr()), 700, C.c_void_p(out.data_ptr()),
                                          700, 700, 600, 4, None)
    assert r == 0, r
    ref = codec.dwt_forward(x, 4, 53, 0)
    assert torch.equal(out, ref)
print("FRESH_OK")
"""


def test_noalloc_first_call_in_a_fresh_process():
    """The first call in a process (the array's address looked up on this device) gives the
    regular transform's output, twice in a row."""
    r = subprocess.run([sys.executable, "-c", _FRESH.format(root=ROOT)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "FRESH_OK" in r.stdout, r.stdout + r.stderr
