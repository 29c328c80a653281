"""Benchmark: Mpixel/s of the Riemersma engines on B200.

Headline workload (`value`, `e2e`): the sequential-exact walk of one
3840x2160 RGB8 frame, 256-colour octree palette, one image per launch (the
plain GPU form), bit-exact with the reference CPU walk.  Synthetic seeded
gradient+noise input (no dataset).  Each step is one full walk.

Also measured and reported in the same JSON line:
  blocks   the block engine on a 4K video batch (fixed palette), GB/s vs HBM
  batched  512 uneven RGBA8 images in one persistent launch vs the plain
           one-launch-per-image form (config 3), with the Amdahl cap
  roofline, cpu_baseline, clocks, e2e, gpu_launches

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one process per GPU, launched by
torch.distributed.run): the images are independent, nothing is exchanged.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HEADLINE = dict(width=3840, height=2160, colors=256, seed=1)
METRIC = "Mpixel/s seq-exact & block engines @4K, batched vs plain; p50/p99 serve latency"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--block-frames", type=int, default=16)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--skip-extra", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=160,
                    help="requests in the served-stream sample (the full stream is 10,000)")
    ap.add_argument("--serve-rates", default="30,120,600",
                    help="Poisson arrival rates (requests/s) of the served-stream sample")
    ap.add_argument("--profile-case", default="none", choices=["none", "seq", "seq_alpha", "blocks", "batched", "jacobi", "frames"],
                    help="run only that workload's device steps (for ncu captures) and print "
                         "its timing; no JSON contract line")
    ap.add_argument("--seq-mode", type=int, default=0, help="profile cases: sequential form")
    ap.add_argument("--size", default="3840x2160", help="profile cases: frame size WxH")
    ap.add_argument("--loop-mode", type=int, default=0,
                    help="profile cases: segmented walk pass loop (1 = host-checked, so ncu "
                         "sees every pass as its own launch; 2 = device-side graph)")
    return ap.parse_args()


# --------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- helpers
def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_cores() -> int:
    return os.cpu_count() or 1


def reference_cpu(img8: np.ndarray, colors: int, budget_s: float):
    """The reference's own RiemersmaWalkCpu (oracle/_ref) or, where that build is
    absent, the C restatement, on the same frame; repeated up to `budget_s`."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from stipple_b200 import synth
    q = synth.to_q16(img8)
    kind = "reference"
    try:
        lib = pyoracle.RefLib()
        run = lambda: lib.walk_seq(q, colors, False, False)  # noqa: E731
    except FileNotFoundError:
        kind = "port"
        orc = pyoracle.Oracle()
        run = lambda: orc.walk_seq(q, colors, False, False)  # noqa: E731
    # Palette build is part of these calls; time it separately and subtract.
    t0 = time.perf_counter()
    if kind == "reference":
        lib.build_tree(q, colors, False, False)
    else:
        orc.build_tree(q, colors, False, False)
    t_tree = time.perf_counter() - t0
    times = []
    start = time.perf_counter()
    while not times or (time.perf_counter() - start < budget_s and len(times) < 20):
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0 - t_tree)
    px = img8.shape[0] * img8.shape[1]
    med = statistics.median(times)
    return {"value": px / med / 1e6, "unit": "Mpixel/s", "cores": 1, "kind": kind,
            "sample": f"{len(times)} sequential walks of the {img8.shape[1]}x{img8.shape[0]} frame "
                      f"({colors} colours), median, palette build excluded"}, times


# --------------------------------------------------------------- main arm
def run_ours(a, rank: int, world: int):
    import torch
    import stipple_b200 as sb
    from stipple_b200 import synth

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    ctx = sb.Context(dev)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    s = stream.cuda_stream
    W, H, C = HEADLINE["width"], HEADLINE["height"], HEADLINE["colors"]
    img = synth.gradient_rgb8(W, H, HEADLINE["seed"] + rank)
    tree = sb.Octree(img, C, False, False)
    pid = ctx.palette_from_octree(tree)
    d_img = torch.from_numpy(img).cuda()
    d_idx = torch.empty((H, W), dtype=torch.uint8, device="cuda")
    job = dict(pixels=d_img.data_ptr(), width=W, height=H, layout=sb.RGB8, palette_id=pid,
               indices=d_idx.data_ptr())
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def step_dev():
        ctx.dither("seq", [job], stream=s)

    # At least five warm-up steps: the segment-length autotuner tries four
    # lengths on its first calls for a workload.
    for _ in range(max(5, a.warmup)):
        step_dev()
    ctx.synchronize(s)
    if world > 1:
        torch.distributed.barrier()
    times = []
    with ClockSampler(dev) as clk:
        for _ in range(a.steps):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step_dev()
            e1.record(stream)
            ctx.synchronize(s)
            times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    # Kernel-level figures: the same step once more with the context's
    # profiling on -- the host then checks each pass and records CUDA events
    # around every walk launch on its stream (the timed steps above run the
    # device-side pass loop, one graph launch, where no event can sit between
    # two of its kernels).  Same kernels, same launches, same passes.
    ctx.profile(True)
    flush.fill_(1)
    step_dev()
    ctx.synchronize(s)
    kstats = ctx.stats()
    ctx.profile(False)
    from stipple_b200 import replicas
    total_ms = replicas.max_over_ranks(sum(times))
    if world > 1:
        torch.distributed.barrier()
    px = W * H
    value = replicas.job_rate(px * a.steps, world, total_ms) / 1e6
    ms_step = total_ms / a.steps

    # Reference-facing call with host buffers: H2D + walk + D2H every step.
    pinned_in = torch.from_numpy(img).pin_memory()
    pinned_out = torch.empty((H, W), dtype=torch.uint8).pin_memory()
    e2e_t = []
    w_e2e = max(5, a.warmup)
    for k in range(w_e2e + a.steps):
        t0 = time.perf_counter()
        ctx.dither_host_into("seq", pinned_in.numpy(), pid, pinned_out.numpy())
        if k >= w_e2e:
            e2e_t.append(time.perf_counter() - t0)
    e2e_ms = replicas.max_over_ranks(sum(e2e_t) * 1e3)
    e2e = {"value": replicas.job_rate(px * len(e2e_t), world, e2e_ms) / 1e6, "unit": "Mpixel/s",
           "h2d_bytes_per_step": int(img.nbytes), "d2h_bytes_per_step": int(W * H)}

    hbm, peak_kind = peaks()
    # Dominant kernel: the segment walk (TswWalkKernel), timed per launch with
    # CUDA events on its stream inside the library.  Algorithmic bytes per
    # walked position: the packed sample (4 B), its uniform-key byte (1 B), its
    # first-touch word (4 B) and the index written (1 B).
    launches = max(1, kstats["walk_launches"])
    walk_ms = kstats["walk_ms"] / launches
    pos_per_launch = kstats["walk_positions"] / launches
    achieved = pos_per_launch * 10 / (walk_ms / 1e3) / 1e9 if walk_ms > 0 else 0.0
    # DRAM bytes of one walk launch of this workload from ncu (dram__bytes_read
    # + dram__bytes_write, pass 30), profiles/tsw_walk_4k_rgb8_256c.md.
    traffic = 64074496 + 4203008
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind,
                "kernel": "TswWalkKernel", "walk_ms_per_launch": walk_ms,
                "positions_per_launch": pos_per_launch,
                "measured_on": "one extra step after the timed ones, host-checked pass loop, "
                               "CUDA events around each walk launch on its stream",
                "note": "each segment is a dependent chain walked by one thread: the kernel "
                        "is bound by the per-step chain latency, not HBM (see chain); DRAM "
                        "traffic per launch is in profiles/"}
    clock = clk.summary()["sm_mhz"]
    seg = int(kstats["seg_len"])
    chain = {"passes_per_step": kstats["passes"], "ns_per_px": ms_step * 1e6 / px,
             "walk_share": kstats["walk_ms"] / (total_ms / a.steps) if total_ms else None,
             "segment_len": seg, "concurrent_chains": int(kstats["chains"]), "clock_mhz": clock}
    if clock and walk_ms > 0 and seg:
        # A launch walks every unverified segment once: seg steps per chain.
        chain["cycles_per_chain_step"] = walk_ms * 1e-3 * clock * 1e6 / seg

    out = {"metric": METRIC, "value": value, "unit": "Mpixel/s", "n_gpus": world,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_step,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded gradient + noise sigma 8, RGB8)",
           "config": {"workload": "seq-exact walk, one 3840x2160 RGB8 frame per launch, "
                                  "256-colour octree palette, bit-exact",
                      "width": W, "height": H, "colors": C, "palette_colors": tree.count,
                      "l2": "flushed between timed steps (256 MB write)",
                      "warmup_steps_run": max(5, a.warmup),
                      "parallelism": f"replicas x{world}"},
           "e2e": e2e, "roofline": roofline, "chain": chain, "clocks": clk.summary(),
           "gpu_launches": int(kstats["launches"]) * a.steps}

    if rank == 0 and not a.skip_extra:
        out["blocks"] = bench_blocks(ctx, s, a, tree, pid, hbm)
        out["batched"] = bench_batched(ctx, s, a)
        out["serve"] = bench_serve(ctx, a)
    if rank == 0:
        cpu, _ = reference_cpu(img, C, budget_s=12.0)
        out["cpu_baseline"] = cpu
    ctx.release_palette(pid)
    return out


def bench_blocks(ctx, s, a, tree, pid, hbm):
    import torch
    import stipple_b200 as sb
    from stipple_b200 import synth
    W, H = HEADLINE["width"], HEADLINE["height"]
    n = a.block_frames
    frames = [torch.from_numpy(synth.video_frame(W, H, 3, f)).cuda() for f in range(n)]
    outs = [torch.empty((H, W), dtype=torch.uint8, device="cuda") for _ in range(n)]
    jobs = [dict(pixels=f.data_ptr(), width=W, height=H, layout=sb.RGB8, palette_id=pid,
                 indices=o.data_ptr()) for f, o in zip(frames, outs)]
    res = {}
    for B in (256, 512, 4096):
        ctx.dither("blocks", jobs, stream=s, block=B)
        ctx.synchronize(s)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.current_stream())
        ctx.dither("blocks", jobs, stream=s, block=B)
        e1.record(torch.cuda.current_stream())
        ctx.synchronize(s)
        ms = e0.elapsed_time(e1)
        px = n * W * H
        gbs = px * 4 / (ms / 1e3) / 1e9
        res[f"B{B}"] = {"ms": ms, "mpx_s": px / ms / 1e3, "gb_s": gbs, "hbm_frac": gbs / hbm}
    res["workload"] = f"{n} frames of 3840x2160 RGB8 video, fixed 256-colour palette"
    res["video_formats"] = bench_frames(ctx, s, a, pid)
    return res


def bench_frames(ctx, s, a, pid):
    """The block engine on the decoder's / encoder's own formats (planar
    4:4:4 in, planar 4:4:4 out: 3 B/px each way) against the RgbaF form the
    reference's callers otherwise convert through (16 B/px each way), B = 512,
    device-timed and end to end through the host-buffer call from pinned
    memory."""
    import torch
    import stipple_b200 as sb
    from stipple_b200 import synth
    W, H = HEADLINE["width"], HEADLINE["height"]
    n = a.block_frames
    yuv = np.stack([synth.yuv444_frame(synth.video_frame(W, H, 3, f)).reshape(-1)
                    for f in range(n)])
    fb = sb.frame_bytes(sb.YUV444P8, W, H)
    d_in = torch.from_numpy(yuv).cuda()
    d_out = torch.empty((n, fb), dtype=torch.uint8, device="cuda")
    res = {"workload": f"{n} frames of 3840x2160, planar YCbCr 4:4:4 in and out, B=512"}
    for _ in range(2):
        ctx.dither_frames(d_in.data_ptr(), sb.YUV444P8, W, H, n, pid, d_out.data_ptr(),
                          sb.YUV444P8, stream=s, block=512)
    ctx.synchronize(s)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(torch.cuda.current_stream())
    ctx.dither_frames(d_in.data_ptr(), sb.YUV444P8, W, H, n, pid, d_out.data_ptr(),
                      sb.YUV444P8, stream=s, block=512)
    e1.record(torch.cuda.current_stream())
    ctx.synchronize(s)
    ms = e0.elapsed_time(e1)
    res["device_mpx_s"] = n * W * H / ms / 1e3
    del d_in, d_out

    def e2e(inp, in_fmt, out_fmt):
        out = torch.empty((n, sb.frame_bytes(out_fmt, W, H)), dtype=torch.uint8).pin_memory()
        ctx.dither_frames_host(inp.numpy(), in_fmt, W, H, pid, out_fmt, out=out.numpy(), block=512)
        t = []
        for _ in range(2):
            t0 = time.perf_counter()
            ctx.dither_frames_host(inp.numpy(), in_fmt, W, H, pid, out_fmt, out=out.numpy(),
                                   block=512)
            t.append(time.perf_counter() - t0)
        return {"mpx_s": n * W * H / min(t) / 1e6, "h2d_bytes": int(inp.numel()),
                "d2h_bytes": int(out.numel())}

    pin_yuv = torch.from_numpy(yuv).pin_memory()
    res["e2e_yuv444"] = e2e(pin_yuv, sb.YUV444P8, sb.YUV444P8)
    del pin_yuv
    rgbaf = torch.empty((n, W * H * 16), dtype=torch.uint8).pin_memory()
    for f in range(n):
        rgbaf[f].numpy().view(np.float32)[:] = synth.to_q16(
            synth.video_frame(W, H, 3, f)).reshape(-1)
    res["e2e_rgbaf"] = e2e(rgbaf, sb.RGBAF32, sb.RGBAF32)
    return res


def bench_batched(ctx, s, a):
    import torch
    import stipple_b200 as sb
    from stipple_b200 import synth
    sizes = synth.log_uniform_sizes(a.batch - 4, seed=2024) + [(1, 1), (3, 5), (17, 13), (4096, 64)]
    rng = np.random.default_rng(5)
    jobs, keep, pids = [], [], []
    for k, (w, h) in enumerate(sizes):
        img = synth.gradient_rgba8(w, h, 1000 + k)
        colors = int(rng.choice([2, 4, 8, 16, 64, 256]))
        pid = ctx.palette_from_image(img, colors, associate_alpha=True)
        d = torch.from_numpy(img).cuda()
        o = torch.empty((h, w), dtype=torch.uint8, device="cuda")
        keep += [d, o]
        pids.append(pid)
        jobs.append(dict(pixels=d.data_ptr(), width=w, height=h, layout=sb.RGBA8, palette_id=pid,
                         indices=o.data_ptr()))
    total = sum(w * h for w, h in sizes)
    biggest = max(w * h for w, h in sizes)
    for _ in range(max(5, a.warmup)):  # the segment-length autotuner explores here
        ctx.dither("seq", jobs, stream=s)
    ctx.synchronize(s)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(torch.cuda.current_stream())
    ctx.dither("seq", jobs, stream=s)
    e1.record(torch.cuda.current_stream())
    ctx.synchronize(s)
    ms_b = e0.elapsed_time(e1)
    t0 = time.perf_counter()
    for j in jobs:
        ctx.dither("seq", [j], stream=s)
        ctx.synchronize(s)
    ms_p = (time.perf_counter() - t0) * 1e3
    for p in pids:
        ctx.release_palette(p)
    return {"images": len(sizes), "total_px": total, "largest_px": biggest,
            "batched_ms": ms_b, "batched_mpx_s": total / ms_b / 1e3,
            "plain_ms": ms_p, "plain_mpx_s": total / ms_p / 1e3,
            "speedup": ms_p / ms_b, "amdahl_cap": total / biggest}


def bench_serve(ctx, a):
    """Served mixed stream (a sample of the 10,000-request stream): Poisson
    arrivals at each rate, W and H log-uniform in 64..4096, RGB8 or RGBA8 (half
    each, alpha-associated palettes for RGBA), colours from {2, 4, ..., 256},
    engines 60 % sequential / 30 % block / 10 % Jacobi, admission capped at
    120 GB.  Latency = submission to result in host memory (palette build,
    admission wait, upload, dither, download).  Beside it, the plain form: the
    same requests one at a time, one call each, on one context."""
    import stipple_b200 as sb
    from stipple_b200 import synth
    rng = np.random.default_rng(77)
    n = a.serve_requests
    sizes = synth.log_uniform_sizes(n, seed=78, lo=64, hi=4096)
    # Requests are crops of two seeded 4096x4096 frames at random offsets (the
    # generator costs ~0.2 us per pixel; cropping keeps the sample cheap).
    base = {False: synth.gradient_rgb8(4096, 4096, 3000), True: synth.gradient_rgba8(4096, 4096, 3001)}
    reqs = []
    for k, (w, h) in enumerate(sizes):
        alpha = bool(rng.random() < 0.5)
        y0 = int(rng.integers(0, 4096 - h + 1))
        x0 = int(rng.integers(0, 4096 - w + 1))
        img = np.ascontiguousarray(base[alpha][y0:y0 + h, x0:x0 + w])
        colors = int(rng.choice([2, 4, 8, 16, 32, 64, 128, 256]))
        u = rng.random()
        engine = "seq" if u < 0.6 else ("blocks" if u < 0.9 else "jacobi")
        reqs.append((img, colors, engine, alpha))
    total_px = sum(w * h for w, h in sizes)
    out = {"requests": n, "total_px": total_px,
           "workload": "served mixed stream sample: sizes log-uniform 64..4096, RGB/RGBA8, "
                       "2..256 colours, 60/30/10 seq/block/Jacobi, 120 GB admission"}
    rates = [float(r) for r in a.serve_rates.split(",") if r]
    for rate in rates:
        srv = sb.Server(budget=120 << 30, workers=4)
        gaps = rng.exponential(1.0 / rate, size=n)
        t0 = time.perf_counter()
        due = t0
        tickets = []
        for (img, colors, engine, alpha), g in zip(reqs, gaps):
            due += g
            now = time.perf_counter()
            if due > now:
                time.sleep(due - now)
            tickets.append(srv.submit(img, colors, engine, alpha=alpha))
        for t in tickets:
            srv.wait(t)
        wall = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        out[f"rate_{rate:g}"] = {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                                 "max_ms": st["max_ms"], "mpx_s": st["mpx_per_s"],
                                 "batches": st["batches"], "wall_s": wall,
                                 "peak_admitted_gb": st["peak_admitted_bytes"] / 2**30}
    # Plain per-request form on the same requests.
    lat = []
    t0 = time.perf_counter()
    for img, colors, engine, alpha in reqs:
        t1 = time.perf_counter()
        tr = sb.Octree(img, colors, alpha)
        pid = ctx.palette_from_octree(tr)
        ctx.dither_host(engine, img, pid)
        ctx.release_palette(pid)
        lat.append((time.perf_counter() - t1) * 1e3)
    plain_s = time.perf_counter() - t0
    out["plain"] = {"mpx_s": total_px / plain_s / 1e6, "p50_ms": float(np.percentile(lat, 50)),
                    "p99_ms": float(np.percentile(lat, 99)), "wall_s": plain_s,
                    "note": "service time per request, no queueing"}
    return out


# ---------------------------------------------------------------- reference arm
def run_reference(a):
    from stipple_b200 import synth
    W, H, C = HEADLINE["width"], HEADLINE["height"], HEADLINE["colors"]
    img = synth.gradient_rgb8(W, H, HEADLINE["seed"])
    for _ in range(max(1, min(a.warmup, 1))):
        reference_cpu(img, C, budget_s=0.0)
    cpu, times = reference_cpu(img, C, budget_s=0.0)
    step_times = []
    for _ in range(a.steps):
        c, t = reference_cpu(img, C, budget_s=0.0)
        step_times.extend(t)
    ms = statistics.median(step_times) * 1e3
    value = W * H / ms / 1e3
    cpu["value"] = value
    return {"metric": METRIC, "value": value, "unit": "Mpixel/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded gradient + noise sigma 8, RGB8)",
            "config": {"workload": "seq-exact walk, one 3840x2160 RGB8 frame, 256-colour octree palette",
                       "width": W, "height": H, "colors": C},
            "impl": "reference", "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": "Mpixel/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def profile_case(a):
    """The device steps of one workload and nothing else: the command the
    ncu summaries under profiles/ were taken with."""
    import torch
    import stipple_b200 as sb
    from stipple_b200 import synth
    torch.cuda.set_device(0)
    ctx = sb.Context(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    s = stream.cuda_stream
    W, H = (int(v) for v in a.size.lower().split("x"))
    C = HEADLINE["colors"]
    img = synth.gradient_rgb8(W, H, HEADLINE["seed"])
    pid = ctx.palette_from_octree(sb.Octree(img, C, False, False))
    if a.profile_case == "batched":
        rng = np.random.default_rng(5)
        sizes = synth.log_uniform_sizes(a.batch - 4, seed=2024) + [(1, 1), (3, 5), (17, 13), (4096, 64)]
        keep, jobs = [], []
        for k, (w, h) in enumerate(sizes):
            im = synth.gradient_rgba8(w, h, 1000 + k)
            p = ctx.palette_from_image(im, int(rng.choice([2, 4, 8, 16, 64, 256])), associate_alpha=True)
            d = torch.from_numpy(im).cuda()
            o = torch.empty((h, w), dtype=torch.uint8, device="cuda")
            keep += [d, o]
            jobs.append(dict(pixels=d.data_ptr(), width=w, height=h, layout=sb.RGBA8, palette_id=p,
                             indices=o.data_ptr()))
        opts = {}
    elif a.profile_case == "frames":
        n = a.block_frames
        yuv = np.stack([synth.yuv444_frame(synth.video_frame(W, H, 3, f)).reshape(-1)
                        for f in range(n)])
        d_in = torch.from_numpy(yuv).cuda()
        d_out = torch.empty_like(d_in)
        for _ in range(a.warmup):
            ctx.dither_frames(d_in.data_ptr(), sb.YUV444P8, W, H, n, pid, d_out.data_ptr(),
                              sb.YUV444P8, stream=s, block=512)
        ctx.synchronize(s)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps):
            ctx.dither_frames(d_in.data_ptr(), sb.YUV444P8, W, H, n, pid, d_out.data_ptr(),
                              sb.YUV444P8, stream=s, block=512)
        e1.record(stream)
        ctx.synchronize(s)
        print(f"frames: {e0.elapsed_time(e1) / max(1, a.steps):.3f} ms per step", flush=True)
        return
    elif a.profile_case in ("seq", "seq_alpha", "jacobi"):
        lay = sb.RGB8
        if a.profile_case == "seq_alpha":
            img = synth.gradient_rgba8(W, H, HEADLINE["seed"])
            pid = ctx.palette_from_image(img, C, associate_alpha=True)
            lay = sb.RGBA8
        d = torch.from_numpy(img).cuda()
        o = torch.empty((H, W), dtype=torch.uint8, device="cuda")
        jobs = [dict(pixels=d.data_ptr(), width=W, height=H, layout=lay, palette_id=pid,
                     indices=o.data_ptr())]
        opts = {"seq_mode": a.seq_mode, "loop_mode": a.loop_mode} if a.profile_case != "jacobi" else {}
    else:
        n = a.block_frames
        frames = [torch.from_numpy(synth.video_frame(W, H, 3, f)).cuda() for f in range(n)]
        outs = [torch.empty((H, W), dtype=torch.uint8, device="cuda") for _ in range(n)]
        jobs = [dict(pixels=f.data_ptr(), width=W, height=H, layout=sb.RGB8, palette_id=pid,
                     indices=x.data_ptr()) for f, x in zip(frames, outs)]
        opts = {"block": 256}
    engine = {"blocks": "blocks", "jacobi": "jacobi"}.get(a.profile_case, "seq")
    for _ in range(a.warmup):
        ctx.dither(engine, jobs, stream=s, **opts)
    ctx.synchronize(s)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        ctx.dither(engine, jobs, stream=s, **opts)
    e1.record(stream)
    ctx.synchronize(s)
    print(f"{a.profile_case}: {e0.elapsed_time(e1) / max(1, a.steps):.3f} ms per step", flush=True)


def main():
    a = parse()
    if a.profile_case != "none":
        profile_case(a)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if a.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(a)), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        torch.distributed.init_process_group(
            "nccl", timeout=datetime.timedelta(seconds=600),
            device_id=torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0"))))
    out = run_ours(a, rank, world)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
