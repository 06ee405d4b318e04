"""Small, self-contained GPU cases for profiling one kernel (or one step) under a profiler.

    python -m roger_b200.profile_cases <case>

Each case builds its inputs, runs the operation once untimed (so that allocations, scratch
buffers and first-launch costs happen before the launch of interest) and then once more;
profile the second run, e.g. ``ncu -k regex:dwt_fwd_fast -s 3 -c 1 ...``.  Sizes follow the
benchmark workloads but stay within a few hundred MB of device memory:

  planar       4096x4096 RGB uint8 -> 3 int32 planes with RCT (1 launch)
  dwt53        level-0 5/3 forward of the three 4096x4096 int32 RCT planes (1 launch per run)
  dwt53-all    6-level 5/3 forward of the same planes
  dwt-px       the encoder's level-0 5/3 forward straight from the 4096x4096 RGB uint8 pixels (tuning
               key J2K_TUNE_DWT_PX; RCT inside the loads, the three components in one launch;
               coefficients only)
  idwt53       level-0 5/3 inverse of the same plane
  tier1        EBCOT tier-1 of one 4096x4096 RCT component (6 levels, 4096 64x64 blocks)
  encode       one whole lossless 4096x4096 RGB encode (planar, 3 x 6 DWT levels, tier-1)
  diff-kernels one level-0 launch of every kernel of the differentiable 9/7 step on
               16 x 1024x1024 float32 (forward, quantiser, inverse+residual, inverse adjoint,
               quantiser backward, forward adjoint+residual)
  diff-step    one fused rate-distortion step (5 levels, forward + backward)
  batched      the 256-image mixed set (config 4) through the batched encoder: the first run
               captures its launch sequence in a CUDA graph, the second replays it
  decode       lossless decode of one 2048x2048 RGB image (tier-1 decode, inverse 5/3, inverse
               RCT) from code-blocks already on the host
  decode-steps / decode-lanes / decode-warp  the same with the tier-1 decoder forced to one
               symbol per step with 32 blocks per warp, to the pass / stripe / column loops with
               8 blocks per warp, or to one warp per block
  decode-4096  the decode case on the 4096x4096 RGB image (12288 code-blocks), default decoder
  rate         one lossless 4096x4096 RGB encode cut to 1 bit per pixel by PCRD-opt (tier-1
               rate path, distortion pass, host PCRD and header sizing, descriptor update)
  dwt53-tma    as dwt53, with the TMA-staged level kernel (tuning key J2K_TUNE_DWT_TMA)
  dwt53-all-tma  as dwt53-all, with the TMA-staged level kernel
  encode-styled  the lossless 4096x4096 RGB encode with code-block style RESET | TERMALL (every
               pass of a block coded in its own lane)
"""
import math
import sys

import torch

from . import codec as C
from . import synth
from ._lib import lib


def _rgb(size=4096):
    return torch.from_numpy(synth.rgb(size, size, (100, 101, 102, 103))).cuda()


def case_planar():
    img = _rgb()
    return lambda: C.rgb_to_planar(img, 1)


def case_dwt53(levels=1):
    planes = C.rgb_to_planar(_rgb(), 1)
    out = torch.empty_like(planes)
    return lambda: C.dwt_forward(planes, levels, out=out)


def case_dwt_px(levels=1):
    img = _rgb()
    ctx = C.Context(0)
    lib().j2k_ctx_set_tuning(ctx.h, 15, 1)  # J2K_TUNE_DWT_PX: level 0 from the pixels
    enc = C.OCLEncoder(ctx=ctx, lossy=False, output_dwt=True)
    return lambda: enc.run_rgb(img, levels=levels)


def _tma(on):
    from ._lib import lib
    lib().j2k_ctx_set_tuning(C.default_context(0).h, 7, 1 if on else 0)


def case_dwt53_tma(levels=1):
    _tma(True)
    return case_dwt53(levels)


def case_encode_styled():
    img = _rgb()
    enc = C.OCLEncoder(lossy=False)
    return lambda: enc.run_rgb(img, levels=6, cbw=64, cbh=64, cblk_style=6)


def case_idwt53():
    planes = C.rgb_to_planar(_rgb(), 1)
    coef = C.dwt_forward(planes[0], 1)
    out = torch.empty_like(coef)
    return lambda: C.dwt_inverse(coef, 1, out=out)


def case_tier1():
    planes = C.rgb_to_planar(_rgb(), 1)
    coef = C.dwt_forward(planes[0], 6)
    bpc = C.OCLBPC()
    return lambda: bpc.run(coef, 6, 64, 64)


def case_encode():
    img = _rgb()
    enc = C.OCLEncoder(lossy=False)
    return lambda: enc.run_rgb(img, levels=6, cbw=64, cbh=64)


def case_diff_kernels():
    from . import diff97 as D
    x = torch.from_numpy(synth.float_batch(16, 1024, 1024, 200)).cuda()
    L = 1
    ls = torch.full((3 * L + 1,), math.log(1 / 64.0), device="cuda")

    def run():
        y = D.dwt97(x, L)
        yh, _, u = D.relaxed_quant(y, ls, L, 200, keep_noise=True)
        d, _ = D.inverse_residual(yh, x, L)
        g = D.idwt97_adjoint(d, L)
        gy, _ = D.relaxed_quant_backward(y, g, ls, L, 200, 0.01, noise=u)
        return D.forward_adjoint_residual(gy, d, L, alpha=1e-3)
    return run


def case_diff_step():
    from . import diff97 as D
    x = torch.from_numpy(synth.float_batch(16, 1024, 1024, 200)).cuda().requires_grad_(True)
    L = 5
    ls = torch.full((3 * L + 1,), math.log(1 / 64.0), device="cuda", requires_grad=True)

    def run():
        x.grad = None
        ls.grad = None
        D.rd_loss(x, ls, L, 0.01, 200).backward()
    return run


def case_batched():
    from .batch import BatchEncoder
    descs = synth.mixed_set(256)
    imgs = [torch.from_numpy(synth.mixed_image(d)).cuda() for d in descs]
    be = BatchEncoder([dict(w=d["w"], h=d["h"], ncomp=d["ncomp"], kernel=d["kernel"], levels=d["levels"],
                            cb=d["cb"]) for d in descs])
    be.encode(imgs)
    return lambda: be.encode(None)


def case_decode(lanes=None, steps=None, size=2048):
    img = synth.rgb(size, size, (100, 101, 102, 103))
    enc = C.OCLEncoder(lossy=False)
    enc.run_rgb(img, levels=6, cbw=64, cbh=64)
    d, b = enc.get_codeblocks()
    dec = C.OCLDecoder(lossy=False)
    if lanes is not None:
        C.check(lib().j2k_ctx_set_tuning(dec.ctx.h, 10, lanes), dec.ctx.h)  # J2K_TUNE_T1D_LANES
    if steps is not None:
        C.check(lib().j2k_ctx_set_tuning(dec.ctx.h, 11, steps), dec.ctx.h)  # J2K_TUNE_T1D_STEPS
    return lambda: dec.run(d, b, size, size, 3, levels=6)


def case_rate():
    img = _rgb()
    enc = C.OCLEncoder(lossy=False)
    return lambda: enc.run_rgb(img, levels=6, cbw=64, cbh=64, target_bytes=4096 * 4096 // 8)


CASES = {"planar": case_planar, "dwt53": case_dwt53, "dwt53-all": lambda: case_dwt53(6), "dwt-px": case_dwt_px,
         "idwt53": case_idwt53, "tier1": case_tier1, "encode": case_encode,
         "diff-kernels": case_diff_kernels, "diff-step": case_diff_step, "batched": case_batched,
         "decode": case_decode,
         "decode-steps": lambda: case_decode(32, 1), "decode-lanes": lambda: case_decode(8, 0),
         "decode-warp": lambda: case_decode(0, 0), "decode-4096": lambda: case_decode(size=4096), "rate": case_rate, "dwt53-tma": case_dwt53_tma,
         "dwt53-all-tma": lambda: case_dwt53_tma(6), "encode-styled": case_encode_styled}


def main(argv):
    if len(argv) != 1 or argv[0] not in CASES:
        print(__doc__)
        print("cases:", ", ".join(CASES))
        return 2
    run = CASES[argv[0]]()
    run()
    torch.cuda.synchronize()
    run()
    torch.cuda.synchronize()
    print("ok", argv[0])
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
