"""Runs oracle encodes on a pool of host processes (test infrastructure only).

The oracle codes about 1.7 Mpix/s on one core, so the full-size parity tests (a 4096x4096 RGB
image, the 256-image mixed set) hand their oracle encodes to one process per host core.  The
pool is started with the "spawn" method, so it is safe after the parent process has used the
GPU.  A job names its input by generator parameters, not by pixels: each worker regenerates the
image from the seeded generator, so nothing large crosses the process boundary.
"""
import multiprocessing as mp
import os
import sys

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _image(job):
    from roger_b200 import synth
    kind = job[0]
    if kind == "rgb":
        _, w, h, seeds = job[:4]
        return synth.rgb(w, h, tuple(seeds))
    if kind == "gray":
        _, w, h, seed = job[:4]
        return synth.gray(w, h, seed)
    if kind == "mixed":
        return synth.mixed_image(job[1])
    raise ValueError(kind)


def encode_job(job):
    """job: ("rgb", w, h, seeds, levels, cb, lossless) | ("gray", w, h, seed, levels, cb,
    lossless) | ("mixed", desc) -> the oracle's codestream bytes."""
    if _ROOT not in sys.path:
        sys.path.insert(0, _ROOT)
    from oracle import oracle as O
    img = _image(job)
    if job[0] == "mixed":
        d = job[1]
        return O.encode_image(img, d["levels"], d["cb"], d["cb"], d["kernel"] == 53)
    levels, cb, lossless = job[4], job[5], job[6]
    return O.encode_image(img, levels, cb, cb, lossless)


def reconstruct_job(desc):
    """The oracle's decode of a lossy (9/7) mixed-set image, as its encoder codes it (colour
    transform ICT for RGB, default steps): the quantised indices dequantised at the interval
    midpoint, the inverse 9/7 and the inverse colour transform -> (H, W[, C]) uint8."""
    if _ROOT not in sys.path:
        sys.path.insert(0, _ROOT)
    import numpy as np
    from oracle import oracle as O
    from roger_b200 import synth
    img = synth.mixed_image(desc)
    L = desc["levels"]
    mct = O.MCT_ICT if desc["ncomp"] == 3 else O.MCT_NONE
    planes = O.planar_fwd(img, mct, as_float=True)
    st = O.default_steps(desc["w"], desc["h"], L)
    rec = O.planar_inv(np.stack([O.dwt97_inv(O.dequantize(O.quantize(O.dwt97_fwd(p, L), L, st), L, st), L)
                                 for p in planes]), mct)
    return rec if desc["ncomp"] == 3 else rec[:, :, 0]


def reconstruct_many(descs, processes=None):
    """reconstruct_job of every descriptor, in order, on a spawned pool of host processes."""
    procs = max(1, min(processes or os.cpu_count() or 1, len(descs)))
    if procs == 1:
        return [reconstruct_job(d) for d in descs]
    with mp.get_context("spawn").Pool(procs) as pool:
        return pool.map(reconstruct_job, descs, chunksize=1)


def encode_many(jobs, processes=None):
    """Oracle codestreams of `jobs`, in order, computed on `processes` host processes (default:
    every core)."""
    procs = max(1, min(processes or os.cpu_count() or 1, len(jobs)))
    if procs == 1:
        return [encode_job(j) for j in jobs]
    # largest first, so that the last jobs to start are short ones
    order = sorted(range(len(jobs)), key=lambda i: -_cost(jobs[i]))
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(encode_job, [jobs[i] for i in order], chunksize=1)
    out = [None] * len(jobs)
    for k, i in enumerate(order):
        out[i] = res[k]
    return out


def _cost(job):
    if job[0] == "mixed":
        return job[1]["w"] * job[1]["h"] * job[1]["ncomp"]
    return job[1] * job[2] * (3 if job[0] == "rgb" else 1)
