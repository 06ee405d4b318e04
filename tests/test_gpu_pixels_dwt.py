"""GPU tests of the first DWT level read straight from interleaved pixels (J2K_TUNE_DWT_PX 1): the
encoder of 8-bit pixels gives the same coefficients and the same code-blocks with it as with the
planar split followed by the DWT of the planes (the default), for gray and colour images,
lossless (RCT + 5/3) and lossy (ICT + 9/7, with and without the quantiser), odd sizes, images
narrower than one tile, and one to six levels; its lossless codestreams equal the oracle's."""
import numpy as np
import pytest

from oracle import oracle as O
from roger_b200 import codec as C
from roger_b200 import synth
from roger_b200._lib import lib

pytestmark = pytest.mark.gpu

TUNE_DWT_PX = 15

SHAPES = [(8, 2), (9, 3), (37, 61), (255, 17), (256, 256), (300, 260), (517, 389), (1000, 33)]


def _ctx(px):
    ctx = C.Context(0)
    assert lib().j2k_ctx_set_tuning(ctx.h, TUNE_DWT_PX, int(px)) == 0
    return ctx


def _img(w, h, nc, seed):
    return synth.rgb(w, h, (seed, seed + 1, seed + 2, seed + 3)) if nc == 3 else synth.gray(w, h, seed)


@pytest.mark.parametrize("w,h", SHAPES)
@pytest.mark.parametrize("nc", [1, 3])
@pytest.mark.parametrize("lossy", [False, True])
def test_pixel_level_matches_planar_split(w, h, nc, lossy):
    img = _img(w, h, nc, 11 + w % 7)
    levels = max(1, min(6, int(np.log2(max(2, min(w, h))))))
    out = {}
    for px in (0, 1):
        enc = C.OCLEncoder(ctx=_ctx(px), lossy=lossy, output_dwt=True)
        out[px] = enc.run_rgb(img, levels=levels).map_dwt_out()
    assert out[1].dtype == out[0].dtype
    assert np.array_equal(out[1].view(np.uint32), out[0].view(np.uint32))


@pytest.mark.parametrize("levels", [1, 2, 3, 6])
@pytest.mark.parametrize("lossy", [False, True])
def test_pixel_level_codeblocks_match_planar_split_and_oracle(levels, lossy):
    img = synth.rgb(333, 270, (21, 22, 23, 24))
    got = {}
    for px in (0, 1):
        enc = C.OCLEncoder(ctx=_ctx(px), lossy=lossy)
        enc.run_rgb(img, levels=levels, cbw=32, cbh=32)
        got[px] = (enc.get_codeblocks(), bytes(enc.codestream()))
    (d0, b0), cs0 = got[0]
    (d1, b1), cs1 = got[1]
    assert np.array_equal(d0, d1) and np.array_equal(b0, b1) and cs0 == cs1
    if not lossy:
        assert cs1 == O.encode_image(img, levels, 32, 32, True)


def test_pixel_level_on_device_input_and_pitch():
    """Device-resident pixels (a CUDA tensor) take the same path and give the host input's result."""
    import torch
    img = synth.rgb(640, 480, (31, 32, 33, 34))
    a = C.OCLEncoder(ctx=_ctx(1)).run_rgb(img, levels=5).get_codeblocks()
    b = C.OCLEncoder(ctx=_ctx(1)).run_rgb(torch.from_numpy(img).cuda(), levels=5).get_codeblocks()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("kernel_dtype", ["int32", "float32"])
def test_dwt_batch_with_odd_plane_strides(kernel_dtype):
    """A batch of planes whose plane stride is odd (even row pitch) transforms like each plane on
    its own: the level kernels keep 8-byte stores and 16-byte copies for batches whose every plane
    stays aligned for them."""
    import torch
    n, h, w, levels = 3, 157, 300, 4
    pitch, stride = w, w * h + 1
    rng = np.random.default_rng(5)
    src = rng.integers(-128, 128, size=(n, h, w)).astype(np.int32)
    dt = torch.int32 if kernel_dtype == "int32" else torch.float32
    flat_in = torch.zeros(n * stride, dtype=dt, device="cuda")
    flat_out = torch.zeros(n * stride, dtype=dt, device="cuda")
    planes = torch.as_strided(flat_in, (n, h, w), (stride, pitch, 1))
    planes.copy_(torch.from_numpy(src).to(dt))
    out = torch.as_strided(flat_out, (n, h, w), (stride, pitch, 1))
    C.dwt_forward(planes, levels, out=out)
    for i in range(n):
        one = C.dwt_forward(planes[i].clone(), levels)  # a fresh, aligned plane
        assert torch.equal(out[i].contiguous().view(torch.int32), one.view(torch.int32))
