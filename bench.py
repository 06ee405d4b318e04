#!/usr/bin/env python3
"""Benchmark: batched JPEG 2000 encode throughput (planar + colour transform -> DWT -> EBCOT
tier-1) on B200, batched against per-image, on the uneven mixed image set.

Headline workload (one "step"): the 256-image mixed set (seed 300): widths and heights
log-uniform in [64, 2048] (odd sizes included), images 0..127 gray and 128..255 RGB uint8,
5/3 lossless with RCT for even and 9/7 FP32 with ICT and dead-zone steps 8*2^-k for odd indices,
3-5 levels by size, 32x32 and 64x64 code-blocks; every image coded to the codewords of its
code-blocks (planar, colour transform, DWT, quantiser, tier-1).  `value` is Mpix/s of the
batched encoder (one CUDA-graph replay per step) with the images resident in HBM; beside it the
same images encoded one OCLEncoder call at a time (`per_image_mpix_s`, `speedup`).  `e2e` is the
same batch from page-locked host images to page-locked host codewords through the C ABI, a
stream of batches with the next batch's upload and the last one's read-back overlapping the
encode.  The 4096x4096 RGB lossless image (the reference's own workload size) is the `c1`
section, and its level-0 DWT launch is the HBM roofline kernel.

Each timed step is bracketed by CUDA events on the launching stream; between steps a 256 MiB
buffer is written and another read to flush L2 (outside the events).  With --gpus N > 1
(torchrun, one rank per GPU) the job is N sets of 256 images (seeds 300 + 1000*s) split over
the ranks by a longest-processing-time partition of whole images (weak scaling, no collective on
the data path); the step time is the max over ranks.  `--impl reference` times the CPU
implementation of the same path (the oracle port of the reference's arithmetic; the reference
itself does not build here) on all host threads, on the same set and the same scope.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "encode Mpix/s (DWT+EBCOT), batched vs per-image on 1 B200, at bit-exact/stated PSNR"
SET_N = 256
SET_SEED = 300
WORKLOAD = ("batched encode of the uneven mixed set: 256 images, w,h log-uniform in [64,2048] (odd sizes "
            "included), 50% gray / 50% RGB uint8, 5/3 lossless + RCT (even index) and 9/7 FP32 + ICT + "
            "dead-zone steps 8*2^-k (odd index), L=3..5, 32x32|64x64 code-blocks; planar + colour transform + "
            "DWT + quantiser + EBCOT tier-1 to every code-block's codeword (no tier-2)")
C1_W = 4096
C1_LEVELS = 6
C1_CB = 64


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--diff", type=int, default=1, help="time the differentiable 9/7 step (1) or not (0)")
    ap.add_argument("--extras", type=int, default=1,
                    help="also time the 4096x4096 sections: lossless encode and decode, lossy, rate control, "
                         "and the 512x512 case (1) or not (0)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------------------------------------
# the workload
# ---------------------------------------------------------------------------------------------

def set_descs(nsets):
    """The image descriptors of `nsets` mixed sets (set s drawn with seed 300 + 1000*s)."""
    from roger_b200 import synth
    out = []
    for s in range(nsets):
        for d in synth.mixed_set(SET_N, seed=SET_SEED + 1000 * s):
            d = dict(d)
            d["set"] = s
            out.append(d)
    return out


def gen_images(descs, threads):
    from roger_b200 import synth
    with ThreadPoolExecutor(max(1, threads)) as ex:
        return list(ex.map(synth.mixed_image, descs))


def mpix_of(descs):
    return sum(d["w"] * d["h"] for d in descs) / 1e6


def config_for(world, descs_all):
    return {"workload": WORKLOAD, "images": len(descs_all), "sets": world, "set_seed": "300 + 1000*s",
            "mpix": round(mpix_of(descs_all), 3),
            "parallelism": "1 GPU" if world == 1 else f"{world} GPUs, whole images split by LPT (no collective "
                                                       "on the data path)",
            "l2": "flushed between timed steps: 256 MiB written, then 256 MiB read"}


# ---------------------------------------------------------------------------------------------
# CPU: the oracle port on host threads
# ---------------------------------------------------------------------------------------------

def cpu_encode_set(descs, images, threads):
    """Wall seconds of the oracle's encode of every image of the set up to its code-blocks'
    codewords (the same scope as the GPU step), on `threads` host threads, largest image first
    (the oracle is C called through ctypes, which releases the GIL).  Returns (seconds, bytes)."""
    from oracle import oracle as O
    order = sorted(range(len(descs)), key=lambda i: -descs[i]["w"] * descs[i]["h"] * descs[i]["ncomp"])

    def one(i):
        d = descs[i]
        return O.encode_tier1(images[i], d["levels"], d["cb"], d["cb"], d["kernel"] == 53)
    with ThreadPoolExecutor(max(1, threads)) as ex:
        t = time.perf_counter()
        total = sum(ex.map(one, order))
        sec = time.perf_counter() - t
    return sec, total


def cpu_baseline(descs, images, threads, passes=1):
    """The oracle on every host thread over the whole set (one warm-up pass over a few images
    first): Mpix/s of the best of `passes` passes."""
    from oracle import oracle as O
    O.lib()
    small = sorted(range(len(descs)), key=lambda i: descs[i]["w"] * descs[i]["h"])[:threads]
    cpu_encode_set([descs[i] for i in small], [images[i] for i in small], threads)
    best = min(cpu_encode_set(descs, images, threads)[0] for _ in range(passes))
    return dict(value=round(mpix_of(descs) / best, 3), unit="Mpix/s", cores=threads, kind="port",
                sample=f"the whole set ({len(descs)} images, {mpix_of(descs):.1f} Mpix): the C oracle's planar + "
                       f"colour transform + DWT + quantiser + tier-1 of every image on {threads} host threads, "
                       f"{best:.2f} s wall clock; images synthesised beforehand")


def cpu_references(tile=1024, reps=2):
    """Single-core CPU figures on one 1024x1024 RGB image of the config-1 kind (no GPU touched):
    the C oracle on one core, and OpenJPEG through Pillow (an independent encoder,
    single-threaded as Pillow drives it) for the lossless 5/3 and the irreversible 9/7 encode."""
    import io
    from oracle import oracle as O
    from roger_b200 import synth
    img = synth.rgb(tile, tile, (100, 101, 102, 103))
    mpix = tile * tile / 1e6

    def best(fn):
        fn()
        tt = []
        for _ in range(reps):
            t = time.perf_counter()
            fn()
            tt.append(time.perf_counter() - t)
        return min(tt)
    out = {"single_thread_oracle": {
        "mpix_s": round(mpix / best(lambda: O.encode_tier1(img, C1_LEVELS, C1_CB, C1_CB, True)), 3),
        "sample": f"one {tile}x{tile} RGB image, RCT+5/3 L={C1_LEVELS}+tier-1"}}
    try:
        from PIL import Image, features
        im = Image.fromarray(img)

        def enc(lossless):
            b = io.BytesIO()
            im.save(b, "JPEG2000", irreversible=not lossless, mct=1, num_resolutions=C1_LEVELS + 1,
                    codeblock_size=(C1_CB, C1_CB), no_jp2=True)
            return b
        out["openjpeg"] = {"version": str(features.version("jpg_2000")), "threads": 1,
                           "lossless_53_mpix_s": round(mpix / best(lambda: enc(True)), 3),
                           "irreversible_97_mpix_s": round(mpix / best(lambda: enc(False)), 3),
                           "sample": f"one {tile}x{tile} RGB image through Pillow, L={C1_LEVELS}, "
                                     f"{C1_CB}x{C1_CB} blocks, colour transform on, tier-2 included"}
    except Exception as e:  # Pillow without OpenJPEG
        out["openjpeg"] = {"unavailable": str(e)[:200]}
    return out


# ---------------------------------------------------------------------------------------------
# profiled figures (ncu summaries kept under profiles/)
# ---------------------------------------------------------------------------------------------

def _profile_values(name, keys):
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    got = {}
    for line in open(path):
        for key in keys:
            if line.startswith(key + ":"):
                got[key] = int(line.split(":")[1])
    return got if len(got) == len(keys) else None


def profiled_traffic(name="dwt_fwd_fast_53_level0_3x4096.txt"):
    """DRAM bytes (read + write) of one launch of a level-0 5/3 kernel on the 4096x4096 RGB image
    (by default the one over the three planes), from the ncu capture of that launch; None when the
    summary is absent."""
    v = _profile_values(name, ["dram_bytes_per_launch"])
    return v["dram_bytes_per_launch"] if v else None


def tier1_issue(profile, kernels, ms, clocks):
    """Issue roofline of tier-1, the dominant stage: its profiled warp instructions (one encode
    of the same workload, deterministic for it) over the live tier-1 time, against the SM issue
    peak (148 SMs x 4 schedulers x 1 instruction per cycle at the SM clock sampled during the
    timed region)."""
    keys = ["t1_symbols_instructions", "t1_mq_instructions"]
    ins = _profile_values(profile, keys)
    if not ins or ms <= 0:
        return None
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    peak = 148 * 4 * mhz * 1e6 / 1e9
    total = ins[keys[0]] + ins[keys[1]]
    achieved = total / (ms * 1e-3) / 1e9
    return {"bound": "issue", "kernels": kernels, "achieved": round(achieved, 1), "peak": round(peak, 1),
            "unit": "G warp-instructions/s", "frac": round(achieved / peak, 4), "instructions_per_encode": total,
            "tier1_ms": round(ms, 4), "source": f"profiles/{profile} (ncu smsp__inst_executed.sum)"}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class L2Flush:
    """Writes a 256 MiB buffer (larger than the 126 MB L2) and then reads another one, so the
    next timed kernel starts with a cold L2 that holds no dirty lines of the flush itself."""

    def __init__(self):
        import torch
        self.a = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        self.b = torch.ones(64 << 20, dtype=torch.int32, device="cuda")

    def fill_(self, v):
        self.a.fill_(v)
        self.s = self.b.sum()
        return self


def ev_once(fn, flush):
    """Device time (ms) of one call of fn, from a cold L2, with CUDA events on the current
    stream."""
    import torch
    flush.fill_(1)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    fn()
    e.record()
    e.synchronize()
    return s.elapsed_time(e)


def ev_median(fn, flush, reps):
    return statistics.median(ev_once(fn, flush) for _ in range(reps))


# ---------------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------------

class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 3 + i and r[3 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------------------------------------
# reference arm: the CPU implementation of the path, same set, same scope
# ---------------------------------------------------------------------------------------------

def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = max(1, os.cpu_count() or 1)
    descs_all = set_descs(world)
    descs = descs_all[:SET_N]  # one set per step (at N > 1 a sample of the N sets)
    images = gen_images(descs, threads)
    base = cpu_baseline(descs, images, threads)  # includes a warm-up pass over a few images
    times = []
    for _ in range(max(1, args.steps)):
        times.append(cpu_encode_set(descs, images, threads)[0])
        if sum(times) > 150.0:  # keep the whole arm within a few minutes
            break
    sec = statistics.median(times)
    v = round(mpix_of(descs) / sec, 3)
    sample = (f"{'the whole set' if world == 1 else f'set 0 of the {world} sets'} per step ({len(descs)} images, "
              f"{mpix_of(descs):.1f} Mpix), the C oracle's planar + colour transform + DWT + quantiser + tier-1 "
              f"of every image on {threads} host threads (wall clock, median of {len(times)} steps)")
    line = dict(metric=METRIC, value=v, unit="Mpix/s", n_gpus=args.gpus, steps=len(times), warmup=args.warmup,
                ms_per_step=round(sec * 1e3, 2), higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="int32/f32", data="synthetic", config=config_for(world, descs_all), impl="reference",
                cpu_baseline=dict(value=v, unit="Mpix/s", cores=threads, kind="port", sample=sample),
                e2e={"value": v, "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                first_pass=base,
                note="the reference (OpenCL 1.2 + Boost + OpenCV, MSVC-only host code, no CPU OpenCL device on the "
                     "box) does not build or run here; this arm times the C oracle that restates its arithmetic "
                     "(completed from T.800 where the reference codes nothing) on all host threads")
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------------

def _enc_desc(d):
    return dict(w=d["w"], h=d["h"], ncomp=d["ncomp"], kernel=d["kernel"], levels=d["levels"], cb=d["cb"])


def dwt_bytes(descs):
    """Algorithmic bytes of the forward DWT of every image of `descs` (4-byte samples in and out
    per level, level k over a quarter^k of the plane), ncomp planes per image."""
    return sum(d["ncomp"] * d["w"] * d["h"] * 8 * sum(4.0 ** -k for k in range(d["levels"])) for d in descs)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank, world, local = dist_env()
    threads = max(1, os.cpu_count() or 1)
    descs_all = set_descs(world)
    from roger_b200 import shard
    mine = shard.shard(descs_all, rank, world)
    descs = [descs_all[i] for i in mine]
    host_imgs = gen_images(descs, threads)
    cpu_line = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_line = cpu_baseline(descs, host_imgs, threads)  # before the first GPU call
        cpu_line.update(cpu_references())
    import numpy as np
    import torch
    from roger_b200 import codec as C
    from roger_b200.batch import BatchEncoder, StreamingBatchEncoder

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=180))
    flush = L2Flush()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def reduce(v, op):
        if world == 1:
            return v
        t = torch.tensor([float(v)], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=op)
        return float(t.item())

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        barrier()
        ms = statistics.mean(ev_once(fn, flush) for _ in range(steps))
        barrier()
        return reduce(ms, torch.distributed.ReduceOp.MAX if world > 1 else None)

    imgs = [torch.from_numpy(im).cuda() for im in host_imgs]
    my_mpix = mpix_of(descs)
    mpix = reduce(my_mpix, torch.distributed.ReduceOp.SUM if world > 1 else None)
    be = BatchEncoder([_enc_desc(d) for d in descs])
    be.encode(imgs)
    tuning = be.autotune(reps=2)
    be.encode(imgs)
    with ClockSampler(local) as clk:
        ms = timed(lambda: be.encode(None), args.steps, args.warmup)
    clocks = clk.summary()
    kernels_per_step = be.get_option(8)

    # stages of the same step, timed apart (planar + DWT, then planar alone)
    def stage_ms(mask):
        be.set_option(9, mask)
        be.encode(None)
        t = ev_median(lambda: be.encode(None), flush, 5)
        be.set_option(9, 7)
        return t
    t_front = stage_ms(3)
    t_planar = stage_ms(1)
    be.encode(None)
    t_tier1 = ms - t_front
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    peak_src = "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s (of fallback)"
    dbytes = dwt_bytes(descs)
    pbytes = sum(d["w"] * d["h"] * d["ncomp"] * 5 for d in descs)  # uint8 in, 4-byte planes out

    # e2e: page-locked host images in, page-locked host codewords out, through the C ABI; a
    # stream of batches (uploads and read-backs overlapping the encodes), steps batches timed
    host = StreamingBatchEncoder.pin(host_imgs)
    in_bytes = sum(h.nbytes for h in host)
    se = StreamingBatchEncoder([_enc_desc(d) for d in descs], depth=2, device=local)
    se.autotune(host)
    for _ in se.run([host] * 3):
        pass
    barrier()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush.fill_(1)
    torch.cuda.synchronize()
    s0.record()
    last = None
    nst = max(3, args.steps)
    for r in se.run([host] * nst):
        last = r
    s1.record()
    s1.synchronize()
    ms_e2e = reduce(s0.elapsed_time(s1) / nst, torch.distributed.ReduceOp.MAX if world > 1 else None)
    out_bytes = sum(int(np.asarray(b).size) + d.nbytes for d, b in last)
    same_stream = all(np.array_equal(d, be.codeblocks(i)[0]) and np.array_equal(np.asarray(b), be.codeblocks(i)[1])
                      for i, (d, b) in enumerate(last))
    del se

    line = dict(
        metric=METRIC, value=round(mpix / (ms * 1e-3), 2), unit="Mpix/s", n_gpus=world, steps=args.steps,
        warmup=args.warmup, ms_per_step=round(ms, 4), higher_is_better=True, scaling="weak", vs_baseline=None,
        dtype="int32/f32", data="synthetic", config=config_for(world, descs_all),
        e2e={"value": round(mpix / (ms_e2e * 1e-3), 2), "unit": "Mpix/s", "h2d_bytes_per_step": int(in_bytes),
             "d2h_bytes_per_step": int(out_bytes), "ms_per_step": round(ms_e2e, 4),
             "path": "StreamingBatchEncoder (j2k_batch_upload, j2k_batch_encode_async, j2k_batch_pack + "
                     "j2k_batch_read_packed): page-locked host images in, every code-block's codeword and "
                     f"descriptor back in page-locked host memory; {nst} batches streamed, the next batch's "
                     "upload and the previous batch's read-back overlapping each encode",
             "identical_to_resident": bool(same_stream)},
        clocks=clocks, gpu_launches=int(args.steps * kernels_per_step), kernels_per_step=int(kernels_per_step),
        tuning=tuning,
        stages_ms={"planar": round(t_planar, 4), "planar_dwt": round(t_front, 4), "tier1": round(t_tier1, 4)},
        batched_dwt={"algorithmic_bytes": int(dbytes), "ms": round(t_front - t_planar, 4),
                     "achieved_gbs": round(dbytes / ((t_front - t_planar) * 1e-3) / 1e9, 1),
                     "frac": round(dbytes / ((t_front - t_planar) * 1e-3) / 1e9 / hbm, 4),
                     "planar_achieved_gbs": round(pbytes / (t_planar * 1e-3) / 1e9, 1),
                     "note": "every DWT launch of the batch (one per level and filter over all images), timed as the "
                             "difference of the planar+DWT and planar-only stage runs"},
        tier1_issue=tier1_issue("tier1_instructions_batched_256_mixed.txt",
                                "t1_symbols_kernel + t1_mq_kernel (batched, tiered warp schedule)", t_tier1, clocks)
        if world == 1 else None,
    )
    if world == 1:
        line.update(bench_per_image(be, descs, imgs, flush, ms, mpix))
    if rank == 0 and args.extras:
        c1 = bench_c1(flush, hbm, peak_src, clocks)
        line["roofline"] = c1.pop("roofline")
        line["c1"] = c1
        img_h = c1.pop("_img_h")
        line["lossless_decode"] = bench_lossless_decode(img_h, c1.pop("_res"), flush)
        st = c1["stages_ms"]
        c1["styles"] = bench_styles(img_h, flush, st["planar_rct"] + st["dwt_all_levels_3comp"], c1["ms_per_step"],
                                    c1["tier1"]["codeword_bytes"])
        if world == 1:
            line["lossy"] = bench_lossy(img_h, flush)
            line["rate_control"] = bench_rate_control(img_h, flush)
            line["c0"] = bench_c0(flush)
            line["batched_decode"] = bench_batched_decode(be, descs, flush)
    if args.diff and world == 1:
        line["diff97"] = bench_diff97(flush, hbm)
    if cpu_line:
        line["cpu_baseline"] = cpu_line
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def bench_styles(img_h, flush, front_ms, plain_ms, plain_bytes):
    """The 4096x4096 lossless encode in the code-block styles that let tier-1 code the passes
    of a block in parallel (context reset + termination after every pass, and that with the
    arithmetic-coding bypass of the low planes' refinement and propagation passes): encode time,
    tier-1 time (encode minus the planar + DWT stages) and the codewords' size against the
    default style."""
    import torch
    from roger_b200 import codec as C
    img_d = torch.from_numpy(img_h).cuda()
    out = {}
    for name, style in (("reset_termall", 6), ("bypass_reset_termall", 7)):
        enc = C.OCLEncoder(lossy=False)

        def step():
            enc.run_rgb(img_d, levels=C1_LEVELS, cbw=C1_CB, cbh=C1_CB, cblk_style=style)
        for _ in range(3):
            step()
        ms = ev_median(step, flush, 7)
        _, data = enc.get_codeblocks()
        nb = int(data.size)
        out[name] = {"cblk_style": style, "ms_per_step": round(ms, 4),
                     "mpix_s": round(img_h.shape[0] * img_h.shape[1] / 1e6 / (ms * 1e-3), 1),
                     "tier1_ms": round(ms - front_ms, 4), "codeword_bytes": nb,
                     "size_vs_default": round(nb / plain_bytes, 4)}
    out["default"] = {"ms_per_step": round(plain_ms, 4), "tier1_ms": round(plain_ms - front_ms, 4),
                      "codeword_bytes": int(plain_bytes)}
    return out


def bench_per_image(be, descs, imgs, flush, ms_batched, mpix):
    """The metric's comparison: the same resident images encoded one OCLEncoder call at a time
    (the reference's one-image-per-run shape, src/OCLEncoder.cpp:43-52), and block-by-block
    identity of the two."""
    import numpy as np
    from roger_b200 import codec as C
    encs = {}

    def per_image():
        for d, im in zip(descs, imgs):
            key = d["kernel"]
            if key not in encs:
                encs[key] = C.OCLEncoder(lossy=key == 97)
            encs[key].run_rgb(im, levels=d["levels"], cbw=d["cb"], cbh=d["cb"])
    per_image()
    t_single = ev_median(per_image, flush, 2)
    same53 = same97 = True
    for i, (d, im) in enumerate(zip(descs, imgs)):
        e = encs[d["kernel"]]
        e.run_rgb(im, levels=d["levels"], cbw=d["cb"], cbh=d["cb"])
        a = e.get_codeblocks()
        b = be.codeblocks(i)
        ok = np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        if d["kernel"] == 53:
            same53 &= ok
        else:
            same97 &= ok
    return {"per_image_ms": round(t_single, 3), "per_image_mpix_s": round(mpix / (t_single * 1e-3), 1),
            "speedup": round(t_single / ms_batched, 2), "bit_identical_53": bool(same53),
            "bit_identical_97": bool(same97), "psnr_delta_db_97": 0.0 if same97 else None}


def bench_c1(flush, hbm, peak_src, clocks):
    """The reference's own workload size: one 4096x4096 RGB lossless encode (RCT + 5/3 L=6 +
    tier-1, 64x64 code-blocks), resident and end to end, with its stages; the level-0 DWT launch
    over the three planes is the HBM roofline kernel.  Beside it, the encoder's other front end:
    the first DWT level reading the interleaved pixels itself (J2K_TUNE_DWT_PX)."""
    import numpy as np
    import torch
    from roger_b200 import codec as C
    from roger_b200 import synth
    size = C1_W
    img_h = synth.rgb(size, size, (100, 101, 102, 103))
    img_d = torch.from_numpy(img_h).cuda()
    img_pinned = torch.from_numpy(img_h).pin_memory()
    enc = C.OCLEncoder(lossy=False)

    def step_device():
        enc.run_rgb(img_d, levels=C1_LEVELS, cbw=C1_CB, cbh=C1_CB)

    def step_e2e():
        enc.run_rgb(img_pinned.numpy(), levels=C1_LEVELS, cbw=C1_CB, cbh=C1_CB)
        return enc.get_codeblocks(pinned=True)
    for _ in range(3):
        step_device()
    ms = statistics.mean(ev_once(step_device, flush) for _ in range(10))
    res = step_e2e()
    d2h = int(res[1].size) + int(res[0].nbytes)
    for _ in range(2):
        step_e2e()
    ms_e2e = statistics.mean(ev_once(step_e2e, flush) for _ in range(5))
    res = step_e2e()
    res = (res[0].copy(), np.array(res[1]))

    planes = C.rgb_to_planar(img_d, 1)
    coef = torch.empty_like(planes)

    def ev_time(fn, reps=5, inner=1):
        """Median over `reps` samples of the device time of `inner` back-to-back calls, per call.
        Each sample starts with a cold L2; the calls inside a sample are queued back to back so
        that the host-side cost of a call overlaps the previous call's kernels (their inputs are
        larger than L2, so nothing is re-read from it)."""
        for _ in range(2):
            fn(0)
        torch.cuda.synchronize()
        return statistics.median(ev_once(lambda: [fn(i) for i in range(inner)], flush) / inner for _ in range(reps))
    imgs4 = [img_d] + [img_d.clone() for _ in range(3)]
    t_planar = ev_time(lambda i: C.rgb_to_planar(imgs4[i % 4], 1), inner=8)
    t_dwt_l0 = ev_time(lambda i: C.dwt_forward(planes, 1, out=coef), inner=8)
    t_dwt = ev_time(lambda i: C.dwt_forward(planes, C1_LEVELS, out=coef), inner=4)
    # the other front end: the DWT from the pixels (coefficients only, no tier-1)
    from roger_b200._lib import lib
    ctx_px = C.Context(0)
    lib().j2k_ctx_set_tuning(ctx_px.h, 15, 1)
    enc_px = C.OCLEncoder(ctx=ctx_px, lossy=False, output_dwt=True)
    t_px_l0 = ev_time(lambda i: enc_px.run_rgb(imgs4[i % 4], levels=1), inner=8)
    t_px = ev_time(lambda i: enc_px.run_rgb(imgs4[i % 4], levels=C1_LEVELS), inner=4)
    n = size * size
    lvl_bytes = sum(n * 8 * 4.0 ** -k for k in range(C1_LEVELS)) * 3
    l0_bytes = 3 * n * 8
    px_l0_bytes = 3 * n + 3 * n * 4  # RGB bytes in, three int32 planes of subbands out
    px_bytes = px_l0_bytes + sum(n * 8 * 4.0 ** -k for k in range(1, C1_LEVELS)) * 3
    achieved = l0_bytes / (t_dwt_l0 * 1e-3) / 1e9
    px_gbs = px_l0_bytes / (t_px_l0 * 1e-3) / 1e9
    descs = res[0]
    samples = int((descs["cw"].astype(np.int64) * descs["ch"] *
                   np.maximum(3 * descs["numbps"].astype(np.int64) - 2, 0)).sum())
    mpix = n / 1e6
    t1_ms = ms - t_planar - t_dwt
    return dict(
        workload=f"lossless encode {size}x{size} RGB uint8: RCT + 5/3 DWT L={C1_LEVELS} + EBCOT tier-1, "
                 f"{C1_CB}x{C1_CB} code-blocks (seeds 100..103), resident",
        mpix_s=round(mpix / (ms * 1e-3), 2), msample_s=round(3 * mpix / (ms * 1e-3), 2), ms_per_step=round(ms, 4),
        e2e={"mpix_s": round(mpix / (ms_e2e * 1e-3), 2), "ms_per_step": round(ms_e2e, 4),
             "h2d_bytes_per_step": int(img_h.nbytes), "d2h_bytes_per_step": d2h,
             "path": "OCLEncoder.run_rgb (j2k_encoder_run_interleaved, pinned host input) + "
                     "get_codeblocks(pinned=True) (device pack + D2H into page-locked buffers)"},
        roofline={"bound": "hbm", "kernel": f"dwt_fwd_fast<53> level 0 (3 x {size}x{size} int32 planes, one launch)",
                  "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                  "traffic": profiled_traffic(), "algorithmic_bytes_per_launch": l0_bytes, "peak_source": peak_src,
                  "workload": "the c1 section's image (4096x4096 RGB, RCT planes)"},
        stages_ms={"planar_rct": round(t_planar, 4), "dwt_all_levels_3comp": round(t_dwt, 4),
                   "dwt_level0_3comp": round(t_dwt_l0, 4), "tier1_all_blocks_derived": round(t1_ms, 4)},
        dwt_from_pixels={"note": "J2K_TUNE_DWT_PX 1: level 0 reads the RGB pixels (level shift and RCT inside its "
                                 "loads), the int32 planes are never written; same coefficients, off by default",
                         "kernel": "dwt_fwd_fast_px<53, 3, RCT> (one launch, a CTA per tile and component)",
                         "level0_ms": round(t_px_l0, 4), "all_levels_ms": round(t_px, 4),
                         "planar_path_front_ms": round(t_planar + t_dwt, 4),
                         "algorithmic_bytes_level0": px_l0_bytes, "level0_gbs": round(px_gbs, 1),
                         "level0_frac": round(px_gbs / hbm, 4),
                         "all_levels_gbs": round(px_bytes / (t_px * 1e-3) / 1e9, 1),
                         "level0_traffic": profiled_traffic("dwt_fwd_fast_px_53_rgb_4096.txt")},
        dwt_all_levels_gbs=round(lvl_bytes / (t_dwt * 1e-3) / 1e9, 1),
        dwt_all_levels_frac=round(lvl_bytes / (t_dwt * 1e-3) / 1e9 / hbm, 4),
        planar_gbs=round(n * 15 / (t_planar * 1e-3) / 1e9, 1),
        planar_frac=round(n * 15 / (t_planar * 1e-3) / 1e9 / hbm, 4),
        tier1_issue=tier1_issue("tier1_instructions_lossless_4096.txt",
                                "t1_symbols_kernel + t1_mq_kernel<16> (tiered warp schedule)", t1_ms, clocks),
        tier1={"codeblocks": int(len(descs)), "sample_passes": samples,
               "gsample_passes_per_s": round(samples / (t1_ms * 1e-3) / 1e9, 3),
               "codeword_bytes": int(res[1].size)},
        _img_h=img_h, _res=res)
def bench_lossless_decode(img_h, res, flush, reps=5):
    """Config 1's round trip: decode the code-blocks of the timed lossless encode (host bytes in,
    host pixels out, through OCLDecoder) and require the exact input back.  Timed three ways:
    with pageable host buffers (wall clock), with page-locked host buffers (CUDA events: the
    35 MB upload, the decode and the 50 MB read-back), and device-resident (the decode kernels
    alone: tier-1, inverse 5/3, inverse RCT)."""
    import ctypes
    import numpy as np
    import torch
    from roger_b200 import codec as C
    from roger_b200._lib import lib
    descs, data = res[0], res[1].cpu().numpy() if hasattr(res[1], "cpu") else res[1]
    h, w, nc = img_h.shape
    dec = C.OCLDecoder(lossy=False)
    out = dec.run(descs, data, w, h, nc, levels=C1_LEVELS, cbw=C1_CB, cbh=C1_CB)
    exact = bool(np.array_equal(out.reshape(img_h.shape), img_h))
    tt = []
    for _ in range(reps):
        t0 = time.perf_counter()
        dec.run(descs, data, w, h, nc, levels=C1_LEVELS, cbw=C1_CB, cbh=C1_CB)
        tt.append(time.perf_counter() - t0)
    t = statistics.median(tt)

    def pinned(nbytes):
        return torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    data_t, descs_t, out_t = pinned(data.size), pinned(descs.nbytes), pinned(h * w * nc)
    data_p = data_t.numpy()
    descs_p = descs_t.numpy().view(descs.dtype)
    out_p = out_t.numpy().reshape(h, w, nc)
    data_p[:] = data
    descs_p[:] = descs

    def run_pinned():
        dec.run(descs_p, data_p, w, h, nc, levels=C1_LEVELS, cbw=C1_CB, cbh=C1_CB, out=out_p)
    run_pinned()
    exact_p = bool(np.array_equal(out_p, img_h))
    ms_p = ev_median(run_pinned, flush, reps)
    descs_d, data_d = descs_t.cuda(), data_t.cuda()
    out_d = torch.empty(h * w * nc, dtype=torch.uint8, device="cuda")
    prm, keep = C._params(C1_LEVELS, C1_CB, C1_CB, 0, None)

    def run_device():
        hh = dec.ctx._bind()
        C.check(lib().j2k_decoder_run_codeblocks(dec.h, ctypes.c_void_p(descs_d.data_ptr()),
                                                 ctypes.c_void_p(data_d.data_ptr()), data.size, 1, nc, w, h,
                                                 ctypes.byref(prm), ctypes.c_void_p(out_d.data_ptr()), 1, w * nc),
                hh)
    run_device()
    exact_d = bool(np.array_equal(out_d.cpu().numpy().reshape(h, w, nc), img_h))
    ms_d = ev_median(run_device, flush, reps)
    return {"workload": "decode of the lossless 4096x4096 RGB encode: tier-1 decode, inverse 5/3 (6 levels), "
                        "inverse RCT, interleave; host code-block bytes in, host pixels out",
            "bit_exact": exact and exact_p and exact_d,
            "ms": round(t * 1e3, 2), "mpix_s": round(w * h / 1e6 / t, 1),
            "page_locked": {"ms": round(ms_p, 3), "mpix_s": round(w * h / 1e3 / ms_p, 1),
                            "h2d_bytes": int(data.size + descs.nbytes), "d2h_bytes": int(h * w * nc),
                            "path": "OCLDecoder.run with page-locked input and output arrays, CUDA events"},
            "device_resident": {"ms": round(ms_d, 3), "mpix_s": round(w * h / 1e3 / ms_d, 1),
                                "path": "j2k_decoder_run_codeblocks on device descriptors, bytes and output"}}


def bench_lossy(img_h, flush, levels=6):
    """Config 2: 4096x4096 RGB, ICT + 9/7 FP32 (6 levels) + dead-zone quantiser (step 8*2^-k at
    level k) + tier-1; encode Mpix/s with the image resident, then decode and reconstruction
    PSNR (the per-subband FP32-vs-FP64 coefficient error is a test: test_c2_fp64_error_per_subband)."""
    import numpy as np
    import torch
    from roger_b200 import codec as C
    h, w, nc = img_h.shape
    img_d = torch.from_numpy(img_h).cuda()
    enc = C.OCLEncoder(lossy=True)

    def step():
        enc.run_rgb(img_d, levels=levels, cbw=C1_CB, cbh=C1_CB)
    for _ in range(2):
        step()
    tt = []
    for _ in range(5):
        flush.fill_(1)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        step()
        e.record()
        e.synchronize()
        tt.append(s.elapsed_time(e))
    ms = statistics.median(tt)
    descs, data = enc.get_codeblocks()
    data = data.cpu().numpy() if hasattr(data, "cpu") else data
    rec = C.OCLDecoder(lossy=True).run(descs, data, w, h, nc, levels=levels, cbw=C1_CB, cbh=C1_CB)
    err = rec.reshape(img_h.shape).astype(np.float64) - img_h.astype(np.float64)
    mse = float((err * err).mean())
    psnr = 10 * math.log10(255.0 ** 2 / mse) if mse > 0 else float("inf")
    return {"workload": f"lossy encode {w}x{h} RGB: ICT + 9/7 FP32 L={levels} + dead-zone steps 8*2^-k + tier-1, "
                        f"{C1_CB}x{C1_CB} code-blocks",
            "ms_per_step": round(ms, 3), "mpix_s": round(w * h / 1e6 / (ms * 1e-3), 1),
            "codeword_bytes": int(data.size if hasattr(data, "size") else len(data)),
            "psnr_db": round(psnr, 3)}


def bench_c0(flush, size=512, levels=5):
    """The reference's CPU-runnable case: one 512x512 gray image (synthetic, seed 0), 5/3 L=5,
    64x64 code-blocks, resident on the device; median of 15 encodes."""
    import torch
    from roger_b200 import codec as C
    from roger_b200 import synth
    img = torch.from_numpy(synth.gray(size, size, 0)).cuda()
    enc = C.OCLEncoder(lossy=False)
    for _ in range(3):
        enc.run_rgb(img, levels=levels, cbw=C1_CB, cbh=C1_CB)
    tt = []
    for _ in range(15):
        flush.fill_(1)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        enc.run_rgb(img, levels=levels, cbw=C1_CB, cbh=C1_CB)
        e.record()
        e.synchronize()
        tt.append(s.elapsed_time(e))
    ms = statistics.median(tt)
    return {"workload": f"{size}x{size} gray uint8, 5/3 L={levels}, {C1_CB}x{C1_CB} code-blocks (seed 0)",
            "ms_per_step": round(ms, 4), "mpix_s": round(size * size / 1e6 / (ms * 1e-3), 1)}


def bench_rate_control(img_h, flush, bpp=1.0):
    """Rate control on config 1's image: lossless pipeline (RCT + 5/3 L=6 + tier-1) with the
    codestream cut to `bpp` bits per pixel by PCRD-opt; encode time with the image resident
    (tier-1 rate path, distortion pass, host PCRD and the descriptor update included), size and
    reconstruction PSNR of the GPU decode."""
    import numpy as np
    import torch
    from roger_b200 import codec as C
    h, w, nc = img_h.shape
    img_d = torch.from_numpy(img_h).cuda()
    target = int(w * h * bpp / 8)
    enc = C.OCLEncoder(lossy=False)

    def step():
        enc.run_rgb(img_d, levels=C1_LEVELS, cbw=C1_CB, cbh=C1_CB, target_bytes=target)
    for _ in range(2):
        step()
    tt = []
    for _ in range(5):
        flush.fill_(1)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        step()
        e.record()
        e.synchronize()
        tt.append(s.elapsed_time(e))
    ms = statistics.median(tt)
    cs = bytes(enc.codestream())
    rec = C.decode_codestream(cs).reshape(img_h.shape)
    err = rec.astype(np.float64) - img_h.astype(np.float64)
    mse = float((err * err).mean())
    return {"workload": f"config-1 image, lossless pipeline cut to {bpp} bpp ({target} bytes) by PCRD-opt",
            "ms_per_step": round(ms, 3), "mpix_s": round(w * h / 1e6 / (ms * 1e-3), 1),
            "codestream_bytes": len(cs), "psnr_db": round(10 * math.log10(255.0 ** 2 / mse), 3)}


def bench_diff97(flush, hbm, n=16, size=1024, levels=5):
    """One rate-distortion training step of the differentiable 9/7 path on 16 x 1024^2 float32
    images (seeds 200..215, /255): forward DWT, relaxed quantiser, inverse DWT, MSE + 0.01 *
    rate, and the backward through the adjoint kernels, for pixels and 16 log-steps.
    Algorithmic traffic of the fused step (every level of this config runs as band kernels, the
    quantiser inside them), N samples of 4 bytes, S = N * sum_{k<L} 4^-k, Nl = N * 4^-(L-1):
    forward with the quantiser (input, y and u of the details, LL): 4 (2.75 S + 0.25 Nl);
    inverse with y_hat formed on load and the residual: 4 (2.75 S + 0.25 Nl + N);
    transpose of the inverse with the quantiser backward (reads y and u): 4 (3.5 S + 0.5 Nl);
    transpose of the forward with the residual term: 4 (2 S + N)."""
    import math
    import numpy as np
    import torch
    from roger_b200 import diff97 as D
    from roger_b200 import synth
    x = torch.from_numpy(synth.float_batch(n, size, size, 200)).cuda().requires_grad_(True)
    ls = torch.full((3 * levels + 1,), math.log(1 / 64.0), device="cuda", requires_grad=True)

    def step():
        x.grad = None
        ls.grad = None
        loss = D.rd_loss(x, ls, levels, 0.01, 200)
        loss.backward()
        return loss

    for _ in range(3):
        step()
    tt = []
    for _ in range(5):
        flush.fill_(1)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        step()
        e.record()
        e.synchronize()
        tt.append(s.elapsed_time(e))
    ms = statistics.median(tt)
    # the same step captured once in a CUDA graph and replayed (no per-kernel host work)
    gstep = D.GraphedRDStep(x, ls, levels, 0.01, 200)
    for _ in range(3):
        gstep()
    tg = []
    for _ in range(5):
        flush.fill_(1)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        gstep()
        e.record()
        e.synchronize()
        tg.append(s.elapsed_time(e))
    ms_graph = statistics.median(tg)
    N = n * size * size
    S = N * sum(4.0 ** -k for k in range(levels))
    Nl = N * 4.0 ** -(levels - 1)
    passes = {"dwt_forward_with_quantiser": int(4 * (2.75 * S + 0.25 * Nl)),
              "dwt_inverse_with_residual": int(4 * (2.75 * S + 0.25 * Nl + N)),
              "dwt_inverse_adjoint_with_quantiser_backward": int(4 * (3.5 * S + 0.5 * Nl)),
              "dwt_forward_adjoint_with_residual": int(4 * (2 * S + N))}
    algo = sum(passes.values())
    return {"workload": f"{n} x {size}x{size} float32, 9/7 L={levels}, relaxed quantiser, loss = MSE + 0.01*rate, "
                        "grads wrt pixels and 16 log-steps",
            "ms_per_step": round(ms, 3), "algorithmic_bytes": int(algo), "algorithmic_bytes_per_pass": passes,
            "achieved_gbs": round(algo / (ms * 1e-3) / 1e9, 1), "hbm_frac": round(algo / (ms * 1e-3) / 1e9 / hbm, 4),
            "mpix_s": round(N / 1e6 / (ms * 1e-3), 1),
            "graphed": {"path": "diff97.GraphedRDStep (the same step captured in one CUDA graph)",
                        "ms_per_step": round(ms_graph, 3),
                        "achieved_gbs": round(algo / (ms_graph * 1e-3) / 1e9, 1),
                        "hbm_frac": round(algo / (ms_graph * 1e-3) / 1e9 / hbm, 4)}}




def bench_batched_decode(be, descs, flush):
    """Batched decode of the set's codestreams (host bytes in, host pixels out, tier-2 parse
    included) against a loop of per-image decodes; 5/3 images must come back exactly."""
    import numpy as np
    from roger_b200 import codec as C
    from roger_b200 import synth
    streams = [be.codestream(i) for i in range(len(descs))]
    dec = C.OCLDecoder()
    outs = C.decode_codestreams(streams, decoder=dec)
    t_b = ev_median(lambda: C.decode_codestreams(streams, decoder=dec), flush, 3)

    def loop():
        return [C.decode_codestream(cs) for cs in streams]
    outs1 = loop()
    t_1 = ev_median(loop, flush, 2)
    mpix = mpix_of(descs)
    same = all(np.array_equal(a.reshape(-1), b.reshape(-1)) for a, b in zip(outs, outs1))
    exact53 = all(np.array_equal(o.reshape(-1), synth.mixed_image(d).reshape(-1))
                  for d, o in zip(descs, outs) if d["kernel"] == 53)
    return {"path": "decode_codestreams (tier-2 of the streams on host threads, one upload, one tier-1 launch, "
                    "per-image inverse DWT + colour transform, one read-back) vs decode_codestream per image",
            "batched_ms": round(t_b, 3), "batched_mpix_s": round(mpix / (t_b * 1e-3), 1),
            "per_image_ms": round(t_1, 3), "per_image_mpix_s": round(mpix / (t_1 * 1e-3), 1),
            "speedup": round(t_1 / t_b, 2), "identical": bool(same), "lossless_exact_53": bool(exact53)}


if __name__ == "__main__":
    sys.exit(main())
