#!/usr/bin/env python3
"""Benchmark: lossless JPEG 2000 encode throughput (planar+RCT -> 5/3 DWT -> EBCOT) on B200.

Workload (one "step"): one 4096x4096 interleaved RGB uint8 image (synthetic, seeds 100..103:
a shared sinusoid field plus per-channel fields and noise, channel correlation ~0.8), RCT,
reversible 5/3 DWT with 6 levels, 64x64 code-blocks, full EBCOT tier-1 encode of all 12,288
code-blocks.  Inputs are resident in HBM when the timed region starts (`value`); `e2e` runs the
same encode through the C ABI from pinned host memory with the code-block bytes read back.

Each timed step is bracketed by CUDA events on the launching stream; between steps a 256 MiB
buffer is written and another read to flush L2 (outside the events).  With --gpus N > 1 (torchrun, one rank per
GPU) every rank encodes its own image (weak scaling, no collective on the data path); the step
time is the max over ranks.  `--impl reference` times the CPU implementation of the same path
(the oracle port of the reference's arithmetic; the reference itself does not build here) on
all host cores over a bounded sample of the same workload.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W = H = 4096
LEVELS = 6
CB = 64
METRIC = "encode Mpix/s (DWT+EBCOT), batched vs per-image on 1 B200, at bit-exact/stated PSNR"
WORKLOAD = "lossless encode 4096x4096 RGB uint8: RCT + 5/3 DWT L=6 + EBCOT tier-1, 64x64 code-blocks"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--size", type=int, default=W, help="image side (default 4096)")
    ap.add_argument("--diff", type=int, default=1, help="time the differentiable 9/7 step (1) or not (0)")
    ap.add_argument("--extras", type=int, default=1,
                    help="also time the config-1 decode round trip and the config-2 lossy encode (1) or not (0)")
    ap.add_argument("--batch-images", type=int, default=256,
                    help="images of the uneven mixed batch timed batched vs per-image (0 = skip)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------------------------------------
# CPU baseline: the oracle port, one process per host core (spawned before any GPU work)
# ---------------------------------------------------------------------------------------------

def _cpu_tile(args):
    size, seeds, levels, cb = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from roger_b200 import synth
    img = synth.rgb(size, size, seeds)
    t = time.perf_counter()
    cs = O.encode_image(img, levels, cb, cb, True)
    return time.perf_counter() - t, len(cs)


def cpu_baseline(tile=1024, tiles=None):
    """Encodes `tiles` independent 1024x1024 RGB images of the workload's kind in parallel, one
    process per host core (about 10 s of encoding in all); returns the encode throughput of all
    cores together (Mpix / (summed per-image encode seconds / processes)) and a description."""
    import multiprocessing as mp
    procs = max(1, os.cpu_count() or 1)
    tiles = tiles or 6 * procs
    ctx = mp.get_context("spawn")
    jobs = [(tile, (100 + 4 * i, 101 + 4 * i, 102 + 4 * i, 103 + 4 * i), LEVELS, CB) for i in range(tiles)]
    with ctx.Pool(procs) as pool:
        pool.map(_cpu_tile, jobs[:procs])  # warm the workers (imports, oracle load)
        t0 = time.perf_counter()
        res = pool.map(_cpu_tile, jobs)
        wall = time.perf_counter() - t0
    busy = sum(r[0] for r in res)
    mpix = tiles * tile * tile / 1e6
    return dict(value=round(mpix / (busy / procs), 3), unit="Mpix/s", cores=procs, kind="port",
                sample=f"{tiles} x {tile}x{tile} RGB images (same generator/parameters), RCT+5/3 L={LEVELS}+"
                       f"tier-1+tier-2 with the C oracle, one process per core; {busy:.1f} s of encoding, "
                       f"wall {wall:.1f} s including input synthesis")


def cpu_references(tile=1024, reps=2):
    """Single-core CPU figures on one tile of the workload's kind (no GPU touched): the C oracle
    on one core, and OpenJPEG through Pillow (an independent encoder, single-threaded as Pillow
    drives it) for the lossless 5/3 and the irreversible 9/7 encode of the same image."""
    import io
    sys.path.insert(0, ROOT)
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
    out = {"single_thread_oracle": {"mpix_s": round(mpix / best(lambda: O.encode_image(img, LEVELS, CB, CB, True)), 3),
                                    "sample": f"one {tile}x{tile} RGB image, RCT+5/3 L={LEVELS}+tier-1+tier-2"}}
    try:
        from PIL import Image, features
        im = Image.fromarray(img)

        def enc(lossless):
            b = io.BytesIO()
            im.save(b, "JPEG2000", irreversible=not lossless, mct=1, num_resolutions=LEVELS + 1,
                    codeblock_size=(CB, CB), no_jp2=True)
            return b
        out["openjpeg"] = {"version": str(features.version("jpg_2000")), "threads": 1,
                           "lossless_53_mpix_s": round(mpix / best(lambda: enc(True)), 3),
                           "irreversible_97_mpix_s": round(mpix / best(lambda: enc(False)), 3),
                           "sample": f"one {tile}x{tile} RGB image through Pillow, L={LEVELS}, {CB}x{CB} blocks, "
                                     "colour transform on"}
    except Exception as e:  # Pillow without OpenJPEG
        out["openjpeg"] = {"unavailable": str(e)[:200]}
    return out


def profiled_traffic(size):
    """DRAM bytes (read + write) of one launch of the level-0 5/3 kernel over the three
    4096x4096 planes, as captured by ncu on the same launch (kept as a text summary under
    profiles/); None when absent or for another size."""
    path = os.path.join(ROOT, "profiles", "dwt_fwd_fast_53_level0_3x4096.txt")
    if size != 4096 or not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch:"):
            return int(line.split(":")[1])
    return None


def tier1_issue(size, ms, clocks):
    """Issue roofline of tier-1, the dominant stage: its profiled warp instructions over the live
    tier-1 time, against the SM issue peak (148 SMs x 4 schedulers x 1 instruction per cycle at
    the SM clock sampled during the timed region)."""
    ins = profiled_tier1_instructions(size)
    if not ins:
        return None
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    peak = 148 * 4 * mhz * 1e6 / 1e9
    total = ins["t1_symbols_instructions"] + ins["t1_mq_instructions"]
    achieved = total / (ms * 1e-3) / 1e9
    return {"bound": "issue", "kernels": "t1_symbols_kernel + t1_mq_kernel<16> (tiered warp schedule)", "achieved": round(achieved, 1),
            "peak": round(peak, 1), "unit": "G warp-instructions/s", "frac": round(achieved / peak, 4),
            "instructions_per_encode": total, "tier1_ms": round(ms, 4),
            "source": "profiles/tier1_instructions_lossless_4096.txt (ncu smsp__inst_executed.sum)"}


def profiled_tier1_instructions(size):
    """Warp instructions of the two tier-1 kernels of one encode of the benchmark image (ncu
    smsp__inst_executed.sum, deterministic for this input; kept as a text summary under
    profiles/); None when absent or for another size."""
    path = os.path.join(ROOT, "profiles", "tier1_instructions_lossless_4096.txt")
    if size != 4096 or not os.path.exists(path):
        return None
    got = {}
    for line in open(path):
        for key in ("t1_symbols_instructions", "t1_mq_instructions"):
            if line.startswith(key + ":"):
                got[key] = int(line.split(":")[1])
    return got if len(got) == 2 else None


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
# reference arm
# ---------------------------------------------------------------------------------------------

def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    cb = cpu_baseline()
    # steps: each step is one bounded sample (wall-clock Mpix/s), as the baseline above
    vals = []
    for _ in range(max(1, min(args.steps, 3))):
        vals.append(cpu_baseline()["value"])
    v = statistics.median(vals)
    line = dict(metric=METRIC, value=v, unit="Mpix/s", n_gpus=args.gpus, steps=len(vals),
                warmup=args.warmup, ms_per_step=None, higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="int32", data="synthetic",
                config={"workload": WORKLOAD + " (CPU sample: 1024x1024 tiles)"},
                impl="reference",
                cpu_baseline=dict(cb, value=v),
                e2e={"value": v, "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                note="the reference (OpenCL 1.2 + Boost + OpenCV, MSVC-only host code) does not build "
                     "here; this arm times the C oracle that restates its arithmetic, on all host cores")
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------------

def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank, world, local = dist_env()
    cpu_line = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_line = cpu_baseline()  # spawned before the first GPU call
        cpu_line.update(cpu_references())
    import numpy as np
    import torch
    from roger_b200 import codec as C
    from roger_b200 import synth

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    size = args.size
    img_h = synth.rgb(size, size, seeds=(100 + 4 * rank, 101 + 4 * rank, 102 + 4 * rank, 103 + 4 * rank))
    img_d = torch.from_numpy(img_h).cuda()
    img_pinned = torch.from_numpy(img_h).pin_memory()
    flush = L2Flush()
    ctx = C.default_context(local)
    enc = C.OCLEncoder(ctx=ctx, lossy=False)

    def step_device():
        enc.run_rgb(img_d, levels=LEVELS, cbw=CB, cbh=CB)

    def step_e2e():
        enc.run_rgb(img_pinned.numpy(), levels=LEVELS, cbw=CB, cbh=CB)
        return enc.get_codeblocks(pinned=True)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        barrier()
        times = []
        for _ in range(steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            e.synchronize()
            times.append(s.elapsed_time(e))
        barrier()
        ms = sum(times) / len(times)
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    with ClockSampler(local) as clk:
        ms = timed(step_device, args.steps, args.warmup)
    clocks = clk.summary()
    res = step_e2e()
    d2h = int(res[1].size) + int(res[0].nbytes)
    ms_e2e = timed(step_e2e, max(3, args.steps // 2), 1)

    # ---- per-stage timing (events on the launching stream), single GPU view
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
        tt = []
        for _ in range(reps):
            flush.fill_(1)
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            for i in range(inner):
                fn(i)
            e.record()
            e.synchronize()
            tt.append(s.elapsed_time(e) / inner)
        return statistics.median(tt)

    # four copies of the image (4 x 50 MB, more than L2 together) cycled by the planar timing
    imgs4 = [img_d] + [img_d.clone() for _ in range(3)]
    t_planar = ev_time(lambda i: C.rgb_to_planar(imgs4[i % 4], 1), inner=8)
    # one launch per level over the three planes (201 MB in, more than L2)
    t_dwt_l0 = ev_time(lambda i: C.dwt_forward(planes, 1, out=coef), inner=8)
    t_dwt = ev_time(lambda i: C.dwt_forward(planes, LEVELS, out=coef), inner=4)

    n = size * size
    lvl_bytes = sum(n * 8 * 4.0 ** -k for k in range(LEVELS)) * 3
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    l0_bytes = 3 * n * 8
    achieved = l0_bytes / (t_dwt_l0 * 1e-3) / 1e9
    descs = res[0]
    samples = int((descs["cw"].astype(np.int64) * descs["ch"] *
                   np.maximum(3 * descs["numbps"].astype(np.int64) - 2, 0)).sum())
    mpix = n / 1e6
    line = dict(
        metric=METRIC, value=round(world * mpix / (ms * 1e-3), 2), unit="Mpix/s",
        msample_s=round(3 * world * mpix / (ms * 1e-3), 2), n_gpus=world,
        steps=args.steps, warmup=args.warmup, ms_per_step=round(ms, 4), higher_is_better=True,
        scaling="weak", vs_baseline=None, dtype="int32", data="synthetic",
        config={"workload": WORKLOAD.replace("4096x4096", f"{size}x{size}"), "levels": LEVELS,
                "codeblock": CB, "images_per_rank": 1, "parallelism": f"replicas x{world} (one image per GPU)",
                "l2": "flushed between timed steps: 256 MiB written, then 256 MiB read"},
        e2e={"value": round(world * mpix / (ms_e2e * 1e-3), 2), "unit": "Mpix/s",
             "h2d_bytes_per_step": int(img_h.nbytes), "d2h_bytes_per_step": d2h,
             "ms_per_step": round(ms_e2e, 4),
             "path": "OCLEncoder.run_rgb (j2k_encoder_run_interleaved, pinned host input) + "
                     "get_codeblocks(pinned=True) (device pack + D2H into page-locked buffers)"},
        roofline={"bound": "hbm", "kernel": f"dwt_fwd_fast<53> level 0 (3 x {size}x{size} int32 planes, one launch)",
                  "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                  "frac": round(achieved / hbm, 4), "traffic": profiled_traffic(size),
                  "algorithmic_bytes_per_launch": l0_bytes,
                  "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback"},
        stages_ms={"planar_rct": round(t_planar, 4), "dwt_all_levels_3comp": round(t_dwt, 4),
                   "dwt_level0_3comp": round(t_dwt_l0, 4),
                   "tier1_all_blocks_derived": round(ms - t_planar - t_dwt, 4)},
        dwt_all_levels_gbs=round(lvl_bytes / (t_dwt * 1e-3) / 1e9, 1),
        planar_gbs=round(n * 15 / (t_planar * 1e-3) / 1e9, 1),
        tier1_issue=tier1_issue(size, ms - t_planar - t_dwt, clocks),
        tier1={"codeblocks": int(len(descs)), "sample_passes": samples,
               "gsample_passes_per_s": round(samples / ((ms - t_planar - t_dwt) * 1e-3) / 1e9, 3),
               "codeword_bytes": int(res[1].size)},
        clocks=clocks,
        # per encode: planar, 3 x 6 DWT levels, tier-1 phase A, the sort's index fill, MQ coder
        gpu_launches=int(args.steps * (1 + 3 * LEVELS + 3)),
    )
    if world == 1 and size == W and args.extras:
        line["lossless_decode"] = bench_lossless_decode(img_h, res)
        line["lossy"] = bench_lossy(img_h, img_d, flush)
        line["rate_control"] = bench_rate_control(img_d, img_h, flush)
        line["c0"] = bench_c0(flush)
    if args.batch_images and world == 1:
        line["batched"] = bench_batched(args.batch_images, flush)
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


def bench_lossless_decode(img_h, res, reps=3):
    """Config 1's round trip: decode the code-blocks of the timed lossless encode (host bytes in,
    host pixels out, through OCLDecoder) and require the exact input back."""
    import numpy as np
    from roger_b200 import codec as C
    descs, data = res[0], res[1].cpu().numpy() if hasattr(res[1], "cpu") else res[1]
    h, w, nc = img_h.shape
    dec = C.OCLDecoder(lossy=False)
    out = dec.run(descs, data, w, h, nc, levels=LEVELS, cbw=CB, cbh=CB)
    tt = []
    for _ in range(reps):
        t0 = time.perf_counter()
        dec.run(descs, data, w, h, nc, levels=LEVELS, cbw=CB, cbh=CB)
        tt.append(time.perf_counter() - t0)
    t = statistics.median(tt)
    return {"workload": "decode of the lossless 4096x4096 RGB encode: tier-1 decode, inverse 5/3 (6 levels), "
                        "inverse RCT, interleave; host code-block bytes in, host pixels out",
            "bit_exact": bool(np.array_equal(out.reshape(img_h.shape), img_h)),
            "ms": round(t * 1e3, 2), "mpix_s": round(w * h / 1e6 / t, 1)}


def bench_lossy(img_h, img_d, flush, levels=6):
    """Config 2: 4096x4096 RGB, ICT + 9/7 FP32 (6 levels) + dead-zone quantiser (step 8*2^-k at
    level k) + tier-1; encode Mpix/s with the image resident, then decode and reconstruction
    PSNR (the per-subband FP32-vs-FP64 coefficient error is a test: test_c2_fp64_error_per_subband)."""
    import numpy as np
    import torch
    from roger_b200 import codec as C
    h, w, nc = img_h.shape
    enc = C.OCLEncoder(lossy=True)

    def step():
        enc.run_rgb(img_d, levels=levels, cbw=CB, cbh=CB)
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
    rec = C.OCLDecoder(lossy=True).run(descs, data, w, h, nc, levels=levels, cbw=CB, cbh=CB)
    err = rec.reshape(img_h.shape).astype(np.float64) - img_h.astype(np.float64)
    mse = float((err * err).mean())
    psnr = 10 * math.log10(255.0 ** 2 / mse) if mse > 0 else float("inf")
    return {"workload": f"lossy encode {w}x{h} RGB: ICT + 9/7 FP32 L={levels} + dead-zone steps 8*2^-k + tier-1, "
                        f"{CB}x{CB} code-blocks",
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
        enc.run_rgb(img, levels=levels, cbw=CB, cbh=CB)
    tt = []
    for _ in range(15):
        flush.fill_(1)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        enc.run_rgb(img, levels=levels, cbw=CB, cbh=CB)
        e.record()
        e.synchronize()
        tt.append(s.elapsed_time(e))
    ms = statistics.median(tt)
    return {"workload": f"{size}x{size} gray uint8, 5/3 L={levels}, {CB}x{CB} code-blocks (seed 0)",
            "ms_per_step": round(ms, 4), "mpix_s": round(size * size / 1e6 / (ms * 1e-3), 1)}


def bench_rate_control(img_d, img_h, flush, bpp=1.0):
    """Rate control on config 1's image: lossless pipeline (RCT + 5/3 L=6 + tier-1) with the
    codestream cut to `bpp` bits per pixel by PCRD-opt; encode time with the image resident
    (tier-1 rate path, distortion pass, host PCRD and the descriptor update included), size and
    reconstruction PSNR of the GPU decode."""
    import numpy as np
    import torch
    from roger_b200 import codec as C
    h, w, nc = img_h.shape
    target = int(w * h * bpp / 8)
    enc = C.OCLEncoder(lossy=False)

    def step():
        enc.run_rgb(img_d, levels=LEVELS, cbw=CB, cbh=CB, target_bytes=target)
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
    Compulsory traffic: 4 transforms of N*8*sum_k 4^-k bytes, quantiser forward 8N, loss and
    its gradient 12N, quantiser backward 12N (N = samples)."""
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
    tr = N * 8 * sum(4.0 ** -k for k in range(levels))
    algo = 4 * tr + 8 * N + 12 * N + 12 * N
    passes = {"dwt_forward": int(tr), "quantiser_forward": int(8 * N), "dwt_inverse_with_residual": int(tr),
              "loss_and_gradient": int(12 * N), "dwt_inverse_adjoint": int(tr), "quantiser_backward": int(12 * N),
              "dwt_forward_adjoint_with_residual": int(tr)}
    return {"workload": f"{n} x {size}x{size} float32, 9/7 L={levels}, relaxed quantiser, loss = MSE + 0.01*rate, "
                        "grads wrt pixels and 16 log-steps",
            "ms_per_step": round(ms, 3), "algorithmic_bytes": int(algo), "algorithmic_bytes_per_pass": passes,
            "achieved_gbs": round(algo / (ms * 1e-3) / 1e9, 1), "hbm_frac": round(algo / (ms * 1e-3) / 1e9 / hbm, 4),
            "mpix_s": round(N / 1e6 / (ms * 1e-3), 1),
            "graphed": {"path": "diff97.GraphedRDStep (the same step captured in one CUDA graph)",
                        "ms_per_step": round(ms_graph, 3),
                        "achieved_gbs": round(algo / (ms_graph * 1e-3) / 1e9, 1),
                        "hbm_frac": round(algo / (ms_graph * 1e-3) / 1e9 / hbm, 4)}}


def bench_batched(n, flush):
    """Uneven mixed set: n images, w,h log-uniform in [64, 2048], half gray / half RGB, 5/3 for
    even and 9/7 (steps 8*2^-k) for odd indices, 3-5 levels, 32x32 / 64x64 code-blocks.  The
    batched encoder (autotuned, graph replay, inputs resident) against a loop of per-image
    encodes of the same device-resident images; results are compared block by block."""
    import numpy as np
    import torch
    from roger_b200 import codec as C
    from roger_b200 import synth
    from roger_b200.batch import BatchEncoder
    descs = synth.mixed_set(n)
    imgs = [torch.from_numpy(synth.mixed_image(d)).cuda() for d in descs]
    mpix = sum(d["w"] * d["h"] for d in descs) / 1e6
    be = BatchEncoder([dict(w=d["w"], h=d["h"], ncomp=d["ncomp"], kernel=d["kernel"], levels=d["levels"],
                            cb=d["cb"]) for d in descs])
    be.encode(imgs)
    tuning = be.autotune(reps=2)
    be.encode(imgs)

    def ev(fn, reps):
        tt = []
        for _ in range(reps):
            flush.fill_(1)
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            e.synchronize()
            tt.append(s.elapsed_time(e))
        return statistics.median(tt)

    for _ in range(3):
        be.encode(None)
    t_batch = ev(lambda: be.encode(None), 5)
    encs = {}

    def per_image():
        for d, im in zip(descs, imgs):
            key = d["kernel"]
            if key not in encs:
                encs[key] = C.OCLEncoder(lossy=key == 97)
            encs[key].run_rgb(im, levels=d["levels"], cbw=d["cb"], cbh=d["cb"])

    per_image()
    t_single = ev(per_image, 2)
    # bit-identity of every image's code-blocks (5/3 and 9/7 alike)
    same53 = same97 = True
    for i, (d, im) in enumerate(zip(descs, imgs)):
        e = C.OCLEncoder(lossy=d["kernel"] == 97)
        e.run_rgb(im, levels=d["levels"], cbw=d["cb"], cbh=d["cb"])
        a = e.get_codeblocks()
        b = be.codeblocks(i)
        ok = np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        if d["kernel"] == 53:
            same53 &= ok
        else:
            same97 &= ok
    # host to host: page-locked host images in, every code-block's codeword back in page-locked
    # host memory (one packing pass per batch).  One batch at a time (copies, encode, copies),
    # then a stream of batches with the next batch's upload and the previous batch's read-back
    # overlapping the current encode (steady-state time per batch).
    from roger_b200.batch import StreamingBatchEncoder
    host = StreamingBatchEncoder.pin([im.cpu().numpy() for im in imgs])
    in_bytes = sum(h.nbytes for h in host)
    se = StreamingBatchEncoder(be.desc, depth=2)
    se.autotune(host)

    def one_batch():
        be.encode(host)
        return be.results(pinned=True)

    for _ in range(3):
        res = one_batch()
    t_seq = ev(one_batch, 5)
    out_bytes = sum(int(np.asarray(b).size) + d.nbytes for d, b in res)
    same_seq = all(np.array_equal(d, be.codeblocks(i)[0]) and np.array_equal(np.asarray(b), be.codeblocks(i)[1])
                   for i, (d, b) in enumerate(res))
    nstream = 8
    for _ in se.run([host] * 3):
        pass
    tt = []
    same_stream = True
    for _ in range(3):
        flush.fill_(1)
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for k, r in enumerate(se.run([host] * nstream)):
            if k == nstream - 1:
                last = r
        s1.record()
        s1.synchronize()
        tt.append(s0.elapsed_time(s1) / nstream)
    for i, (d, b) in enumerate(last):
        rd, rb = be.codeblocks(i)
        same_stream &= np.array_equal(d, rd) and np.array_equal(np.asarray(b), rb)
    t_stream = statistics.median(tt)
    # batched decode of the same 256 codestreams (host bytes in, host pixels out, tier-2 parse
    # included) against a loop of per-image decodes
    streams = [be.codestream(i) for i in range(len(descs))]
    dec = C.OCLDecoder()
    outs = C.decode_codestreams(streams, decoder=dec)
    t_dec_b = ev(lambda: C.decode_codestreams(streams, decoder=dec), 3)

    def dec_loop():
        return [C.decode_codestream(cs) for cs in streams]
    outs1 = dec_loop()
    t_dec_1 = ev(dec_loop, 2)
    dec_same = all(np.array_equal(a.reshape(-1), b.reshape(-1)) for a, b in zip(outs, outs1))
    exact53 = all(np.array_equal(o.reshape(-1), im.cpu().numpy().reshape(-1))
                  for d, o, im in zip(descs, outs, imgs) if d["kernel"] == 53)
    decode = {"path": "decode_codestreams (tier-2 of the streams on host threads, one upload, one tier-1 "
                      "launch, per-image inverse DWT + colour transform, one read-back) vs decode_codestream per "
                      "image",
              "batched_ms": round(t_dec_b, 3), "batched_mpix_s": round(mpix / (t_dec_b * 1e-3), 1),
              "per_image_ms": round(t_dec_1, 3), "per_image_mpix_s": round(mpix / (t_dec_1 * 1e-3), 1),
              "speedup": round(t_dec_1 / t_dec_b, 2), "identical": bool(dec_same), "lossless_exact_53": bool(exact53)}
    h2h = {"h2d_bytes_per_batch": in_bytes, "d2h_bytes_per_batch": out_bytes,
           "one_batch": {"ms": round(t_seq, 3), "mpix_s": round(mpix / (t_seq * 1e-3), 1),
                         "identical_to_batched": bool(same_seq)},
           "streamed": {"batches": nstream, "ms_per_batch": round(t_stream, 3),
                        "mpix_s": round(mpix / (t_stream * 1e-3), 1), "identical_to_batched": bool(same_stream)}}
    return {"workload": f"{n} images, w,h log-uniform [64,2048], 50% RGB, 5/3 even / 9/7 odd, L=3..5, "
                        "32x32|64x64 code-blocks (seed 300)",
            "host_to_host": h2h, "decode": decode,
            "mpix": round(mpix, 3), "batched_ms": round(t_batch, 3), "per_image_ms": round(t_single, 3),
            "batched_mpix_s": round(mpix / (t_batch * 1e-3), 1),
            "per_image_mpix_s": round(mpix / (t_single * 1e-3), 1),
            "speedup": round(t_single / t_batch, 2), "tuning": tuning,
            "bit_identical_53": bool(same53), "bit_identical_97": bool(same97),
            "psnr_delta_db_97": 0.0 if same97 else None}


if __name__ == "__main__":
    sys.exit(main())
