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
# Algorithmic bytes per pixel of the path: 3 B RGB8 sample in, 1 B index out.
ALG_BYTES_PER_PX = 4
# Untimed calls before a timed region: the segment-length tuner's untimed
# first call and one timed call per candidate (four) settle in them, with
# room to spare.
WARM_CALLS = 7
# DRAM bytes (read + write) of one walk launch of the 4K walk in its default
# form (TswWalkPairKernel: 96-position segments, a window of the resident
# ones), from one ncu capture (profiles/tsw_walk_pair_4k_rgb8_256c.md).
TSW_TRAFFIC_PER_LAUNCH = 37494784 + 871168
# The per-step dependent path of the thread walker, as a sum of measured
# latencies (rdb_probe_latency on the same GPU): the head's DMUL and DADD,
# double -> float (clamp), float -> int and the byte rule's integer ops, the
# key's integer ops, the uniform-key table load as an L1 hit, the
# shared-memory colour load, float -> double and the residual's DADD.
BYTE_INT_OPS = 4   # add 257, divide by 514 (multiply-high and shift), min 255
KEY_INT_OPS = 3    # shift, shift-or, or


def chain_path_cycles(lat: dict) -> float:
    return (lat["dmul"] + lat["dadd"] + lat["f64_to_f32"] + lat["f32_to_int"] +
            (BYTE_INT_OPS + KEY_INT_OPS) * lat["int_op"] + lat["global_load_l1"] +
            lat["shared_load"] + lat["f32_to_f64"] + lat["dadd"])


CHAIN_LATENCY_SOURCE = "rdb_probe_latency, measured in this run (profiles/chain_latency_table.md)"
METRIC = "Mpixel/s seq-exact & block engines @4K, batched vs plain; p50/p99 serve latency"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--block-frames", type=int, default=16,
                    help="frames of the video-format (4:4:4) block measurement")
    ap.add_argument("--block-clip", type=int, default=120,
                    help="frames of the block engine's video clip")
    ap.add_argument("--block-sweep", default="256,1024,4096,16384,65536",
                    help="block lengths of the block engine's sweep")
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--skip-extra", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=2000,
                    help="requests of the served stream at each rate")
    ap.add_argument("--serve-rates", default="60,240,1000",
                    help="Poisson arrival rates (requests/s) of the served stream")
    ap.add_argument("--serve-stream", type=int, default=0,
                    help="also run a stream of this many requests (10000: the full stream) "
                         "at the last rate")
    ap.add_argument("--cpu-serve-requests", type=int, default=300,
                    help="served-stream requests in the all-cores CPU sample")
    ap.add_argument("--serve-plain", type=int, default=300,
                    help="requests of the plain one-at-a-time form")
    ap.add_argument("--profile-case", default="none", choices=["none", "seq", "seq_alpha", "blocks", "batched", "jacobi", "frames"],
                    help="run only that workload's device steps (for ncu captures) and print "
                         "its timing; no JSON contract line")
    ap.add_argument("--seq-mode", type=int, default=0, help="profile cases: sequential form")
    ap.add_argument("--walk-form", type=int, default=0,
                    help="profile cases: segmented walk form (1 paired warps, 2 one thread a segment)")
    ap.add_argument("--seg-len", type=int, default=0, help="profile cases: segment length (0 = tuned)")
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
    q1, q3 = (float(v) for v in np.percentile(times, [25, 75]))
    return {"value": px / med / 1e6, "unit": "Mpixel/s", "cores": 1, "kind": kind,
            "cpu_model": cpu_model(), "host_cpus": os.cpu_count(),
            "iqr_mpx_s": [px / q3 / 1e6, px / q1 / 1e6], "runs": len(times),
            "sample": f"{len(times)} sequential walks of the {img8.shape[1]}x{img8.shape[0]} frame "
                      f"({colors} colours), median, palette build excluded; the walk is one "
                      f"dependent chain, so one thread"}, times


# Synthetic inputs that several measurements share, generated once.
_CACHE: dict = {}


def mixed_batch_images():
    """The mixed-size batch (synth.mixed_batch_spec) as RGBA8 arrays."""
    from stipple_b200 import synth
    if "batch" not in _CACHE:
        spec = synth.mixed_batch_spec(512)
        _CACHE["batch"] = (spec, [synth.gradient_rgba8(w, h, seed) for w, h, seed, _ in spec])
    return _CACHE["batch"]


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_all_cores(a, img8: np.ndarray, colors: int, serve_rates):
    """The reference's own CPU engines (oracle/_ref) on every host CPU this
    process may use, one independent image per thread (the walks release the
    GIL): the 4K frame, the mixed-size batch, a video frame in block mode, and
    a sample of the served stream with palette builds, whose measured service
    times are replayed through a FIFO queue of `cores` servers at each
    arrival rate (a host-only server's p50/p99, simulated from measured
    service times).  Bounded samples; figures in Mpixel/s."""
    from concurrent.futures import ThreadPoolExecutor
    import ctypes as C
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from stipple_b200 import synth
    try:
        lib = pyoracle.RefLib()
    except FileNotFoundError:
        return {"unavailable": "oracle/_ref (the reference's CPU build) is not present"}
    raw = lib.lib
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)

    def walk(q, colors_, assoc, block=0):
        """Palette build (untimed) then one walk (timed); returns seconds."""
        h, w = q.shape[:2]
        px = np.ascontiguousarray(q, dtype=np.float32).reshape(-1)
        t = raw.ref_tree_build(px, w, h, int(colors_), int(assoc), int(synth.is_grayscale(q[..., :3])))
        try:
            out = px.copy()
            t0 = time.perf_counter()
            if block:
                err = C.create_string_buffer(256)
                raw.ref_walk_blocks(t, 1.0, int(block), w, h, out, 1, err, 256)
            else:
                raw.ref_walk_seq(t, 1.0, 1, w, h, out)
            return time.perf_counter() - t0
        finally:
            raw.ref_tree_free(t)

    def pool(fn, items):
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=cores) as ex:
            res = list(ex.map(fn, items))
        return time.perf_counter() - t0, res

    res = {"cores": cores}
    q4k = synth.to_q16(img8)
    wall, _ = pool(lambda _: walk(q4k, colors, False), range(cores))
    res["frames_4k"] = {"mpx_s": cores * img8.shape[0] * img8.shape[1] / wall / 1e6,
                        "sample": f"{cores} walks of the 3840x2160 frame, one per thread"}
    spec, imgs8 = mixed_batch_images()
    imgs = [synth.to_q16(im) for im in imgs8]
    order = sorted(range(len(spec)), key=lambda i: -imgs[i].shape[0] * imgs[i].shape[1])
    wall, _ = pool(lambda i: walk(imgs[i], spec[i][3], True), order)
    total = sum(q.shape[0] * q.shape[1] for q in imgs)
    res["batched"] = {"mpx_s": total / wall / 1e6, "wall_s": wall,
                      "sample": "the 512-image mixed RGBA8 batch, images spread over the threads "
                                "largest first, palette builds outside the walk time"}
    del imgs
    vq = synth.to_q16(synth.video_frame(3840, 2160, 3, 0))
    wall, _ = pool(lambda _: walk(vq, 256, False, block=256), range(cores))
    res["blocks_4k_b256"] = {"mpx_s": cores * 3840 * 2160 / wall / 1e6,
                             "sample": f"{cores} block-mode walks (B = 256) of a 4K video frame"}
    # Served stream sample: service = palette build + the request's engine
    # (RiemersmaBlocksCpu for block requests, RiemersmaWalkCpu otherwise: the
    # reference has no CPU form of the approximation).
    reqs, _ = serve_requests(a.cpu_serve_requests, seed=77)

    def service(r):
        img, colors_, engine, alpha = r
        q = synth.to_q16(np.ascontiguousarray(img))
        t0 = time.perf_counter()
        if engine == "blocks":
            lib.walk_blocks(q, colors_, alpha, synth.is_grayscale(img[..., :3]), 256)
        else:
            lib.walk_seq(q, colors_, alpha, synth.is_grayscale(img[..., :3]))
        return time.perf_counter() - t0

    wall, svc = pool(service, reqs)
    px = sum(r[0].shape[0] * r[0].shape[1] for r in reqs)
    served = {"requests": len(reqs), "saturated_mpx_s": px / wall / 1e6,
              "service_p50_ms": float(np.percentile(svc, 50)) * 1e3,
              "service_p99_ms": float(np.percentile(svc, 99)) * 1e3,
              "sample": f"first {len(reqs)} requests of the served stream, palette build "
                        f"included, {cores} threads"}
    for k, rate in enumerate(serve_rates):
        gaps = np.random.default_rng(100 + k).exponential(1.0 / rate, size=len(reqs))
        free = [0.0] * cores
        lat = []
        now = 0.0
        for g, sv in zip(gaps, svc):
            now += g
            j = min(range(cores), key=lambda i: free[i])
            start = max(now, free[j])
            free[j] = start + sv
            lat.append(free[j] - now)
        served[f"rate_{rate:g}"] = {"p50_ms": float(np.percentile(lat, 50)) * 1e3,
                                    "p99_ms": float(np.percentile(lat, 99)) * 1e3,
                                    "note": "FIFO queue of `cores` servers replayed with the "
                                            "measured service times"}
    res["served"] = served
    return res


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
    for _ in range(max(WARM_CALLS, a.warmup)):
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
    w_e2e = max(WARM_CALLS, a.warmup)
    for k in range(w_e2e + a.steps):
        t0 = time.perf_counter()
        ctx.dither_host_into("seq", pinned_in.numpy(), pid, pinned_out.numpy())
        if k >= w_e2e:
            e2e_t.append(time.perf_counter() - t0)
    e2e_ms = replicas.max_over_ranks(sum(e2e_t) * 1e3)
    e2e = {"value": replicas.job_rate(px * len(e2e_t), world, e2e_ms) / 1e6, "unit": "Mpixel/s",
           "h2d_bytes_per_step": int(img.nbytes), "d2h_bytes_per_step": int(W * H)}

    hbm, peak_kind = peaks()
    # Dominant kernel: the segment walk (TswWalkPairKernel), timed per launch with
    # CUDA events on its stream inside the library.  Algorithmic bytes are
    # those of the path itself: 3 B of RGB8 sample in and 1 B of index out per
    # pixel (4 B/px).  A launch walks `pos_per_launch` positions, so per launch
    # the algorithmic traffic is 4 B x positions; per frame it is 4 B x pixels.
    launches = max(1, kstats["walk_launches"])
    walk_ms = kstats["walk_ms"] / launches
    pos_per_launch = kstats["walk_positions"] / launches
    achieved = pos_per_launch * ALG_BYTES_PER_PX / (walk_ms / 1e3) / 1e9 if walk_ms > 0 else 0.0
    frame_gbs = px * ALG_BYTES_PER_PX / (ms_step / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": TSW_TRAFFIC_PER_LAUNCH, "peak_kind": peak_kind,
                "kernel": "TswWalkPairKernel", "walk_ms_per_launch": walk_ms,
                "positions_per_launch": pos_per_launch,
                "algorithmic_bytes_per_px": ALG_BYTES_PER_PX,
                "per_frame": {"algorithmic_bytes": px * ALG_BYTES_PER_PX, "ms": ms_step,
                              "gb_s": frame_gbs, "frac": frame_gbs / hbm},
                "traffic_breakdown": {
                    "scratch_bytes_per_walked_position": 10,
                    "parts": "packed sample 4, uniform-key byte 1, first-touch word 4, index byte 1",
                    "ncu_dram_bytes_per_launch": TSW_TRAFFIC_PER_LAUNCH,
                    "source": "profiles/tsw_walk_pair_4k_rgb8_256c.md"},
                "measured_on": "one extra step after the timed ones, host-checked pass loop, "
                               "CUDA events around each walk launch on its stream",
                "note": "each segment is a dependent chain walked by a chain warp's lane, its "
                        "running sums kept by a paired warp: the kernel is bound by the per-step "
                        "chain latency, not HBM (see chain)"}
    clock = clk.summary()["sm_mhz"]
    lat = sb.probe_latency(dev)
    path_cycles = chain_path_cycles(lat)
    seg = int(kstats["seg_len"])
    chains = int(kstats["chains"])
    chain = {"passes_per_step": kstats["passes"], "ns_per_px": ms_step * 1e6 / px,
             "walk_share": kstats["walk_ms"] / (total_ms / a.steps) if total_ms else None,
             "segment_len": seg, "concurrent_chains": chains, "clock_mhz": clock,
             "walked_positions_per_px": kstats["walk_positions"] / px,
             "latency_table": lat, "latency_source": CHAIN_LATENCY_SOURCE,
             "dependent_path_cycles": path_cycles}
    if clock and walk_ms > 0 and seg:
        # A launch walks every unverified segment once: seg steps per chain.
        chain["cycles_per_chain_step"] = walk_ms * 1e-3 * clock * 1e6 / seg
        # The bound: every resident chain advancing one step per dependent-path
        # latency.  Per launch: walked positions / launch time against it; per
        # frame: the frame's pixels / step time against it.
        bound = chains * clock * 1e6 / path_cycles
        chain["bound_steps_per_s"] = bound
        chain["achieved_steps_per_s"] = pos_per_launch / (walk_ms / 1e3)
        chain["frac"] = chain["achieved_steps_per_s"] / bound
        chain["frame_steps_per_s"] = px / (ms_step / 1e3)
        chain["frame_frac"] = chain["frame_steps_per_s"] / bound

    # The same walk at 1920x1080 (the second frame size of the plain form).
    fhd = _side(bench_frame_size, ctx, s, a, 1920, 1080)
    # The call the reference's RiemersmaWalkCuda makes: RgbaF Q16 frame in a
    # host buffer, dithered in place (16 B/px each way), through the host C ABI.
    rgbaf = _side(bench_rgbaf_inplace, ctx, a, img, pid)

    out = {"metric": METRIC, "value": value, "unit": "Mpixel/s", "n_gpus": world,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_step,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded gradient + noise sigma 8, RGB8)",
           "config": {"workload": "seq-exact walk, one 3840x2160 RGB8 frame per launch, "
                                  "256-colour octree palette, bit-exact",
                      "width": W, "height": H, "colors": C, "palette_colors": tree.count,
                      "l2": "flushed between timed steps (256 MB write)",
                      "warmup_steps_run": max(WARM_CALLS, a.warmup),
                      "parallelism": f"replicas x{world}"},
           "e2e": e2e, "roofline": roofline, "chain": chain, "clocks": clk.summary(),
           "config2_1080p": fhd, "e2e_rgbaf_inplace": rgbaf,
           "gpu_launches": int(kstats["launches"]) * a.steps}

    if rank == 0 and not a.skip_extra:
        out["blocks"] = _side(bench_blocks, ctx, s, a, tree, pid, hbm)
        out["batched"] = _side(bench_batched, ctx, s, a)
        out["serve"] = _side(bench_serve, ctx, a)
    if rank == 0:
        cpu, _ = reference_cpu(img, C, budget_s=12.0)
        if not a.skip_extra:
            cpu["all_cores"] = _side(cpu_all_cores, a, img, C,
                                     [float(r) for r in a.serve_rates.split(",") if r])
        out["cpu_baseline"] = cpu
    ctx.release_palette(pid)
    return out


def _side(fn, *args):
    """A side measurement: its failure is recorded in the line (and its
    traceback on stderr) instead of losing the headline."""
    try:
        return fn(*args)
    except Exception as exc:  # noqa: BLE001 -- reported, not swallowed
        import traceback
        traceback.print_exc(file=sys.stderr)
        return {"error": f"{type(exc).__name__}: {exc}"}


def bench_frame_size(ctx, s, a, W, H):
    """The headline walk at another frame size: device-timed (inputs resident,
    L2 flushed between steps) and end to end through the host-buffer call."""
    import torch
    import stipple_b200 as sb
    from stipple_b200 import synth
    img = synth.gradient_rgb8(W, H, HEADLINE["seed"])
    pid = ctx.palette_from_octree(sb.Octree(img, HEADLINE["colors"], False, False))
    d_img = torch.from_numpy(img).cuda()
    d_idx = torch.empty((H, W), dtype=torch.uint8, device="cuda")
    job = dict(pixels=d_img.data_ptr(), width=W, height=H, layout=sb.RGB8, palette_id=pid,
               indices=d_idx.data_ptr())
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    for _ in range(max(WARM_CALLS, a.warmup)):
        ctx.dither("seq", [job], stream=s)
    ctx.synchronize(s)
    times = []
    for _ in range(max(3, a.steps)):
        flush.fill_(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.dither("seq", [job], stream=s)
        e1.record(stream)
        ctx.synchronize(s)
        times.append(e0.elapsed_time(e1))
    pin_in = torch.from_numpy(img).pin_memory()
    pin_out = torch.empty((H, W), dtype=torch.uint8).pin_memory()
    t = []
    for k in range(3 + max(3, a.steps)):
        t0 = time.perf_counter()
        ctx.dither_host_into("seq", pin_in.numpy(), pid, pin_out.numpy())
        if k >= 3:
            t.append(time.perf_counter() - t0)
    ctx.release_palette(pid)
    ms = sum(times) / len(times)
    return {"workload": f"seq-exact walk, one {W}x{H} RGB8 frame per launch, 256 colours",
            "value": W * H / ms / 1e3, "unit": "Mpixel/s", "ms_per_step": ms,
            "passes": ctx.last_passes,
            "e2e": {"value": W * H * len(t) / sum(t) / 1e6, "unit": "Mpixel/s",
                    "h2d_bytes_per_step": int(img.nbytes), "d2h_bytes_per_step": W * H}}


def bench_rgbaf_inplace(ctx, a, img8, pid):
    """What the reference-facing RiemersmaWalkCuda(..., RgbaF* pixels, ...) does
    per call: an RgbaF Q16 frame in host memory (pinned), dithered in place,
    16 B/px up and 16 B/px down (plus the 1 B/px index map the C ABI always
    returns), through the host C ABI the drop-in calls."""
    import torch
    from stipple_b200 import synth
    H, W = img8.shape[:2]
    q = torch.from_numpy(synth.to_q16(img8)).pin_memory()
    buf = torch.empty_like(q).pin_memory()
    idx = torch.empty((H, W), dtype=torch.uint8).pin_memory()
    t = []
    for k in range(3 + max(3, a.steps)):
        buf.copy_(q)  # a fresh frame each call (outside the timed region)
        t0 = time.perf_counter()
        ctx.dither_host_into("seq", buf.numpy(), pid, idx.numpy(), rgba_out=buf.numpy())
        if k >= 3:
            t.append(time.perf_counter() - t0)
    return {"value": W * H * len(t) / sum(t) / 1e6, "unit": "Mpixel/s",
            "h2d_bytes_per_step": W * H * 16, "d2h_bytes_per_step": W * H * 17,
            "workload": f"seq-exact walk of one {W}x{H} RgbaF (Q16 float4) frame in place"}


def bench_blocks(ctx, s, a, tree, pid, hbm):
    """The block engine on the video clip: `block_clip` frames of 3840x2160
    RGB8 (gradients translating 2 px a frame plus fresh noise sigma 6 each
    frame, generated on the device), one fixed 256-colour palette, every
    frame in one call, for each block length of the sweep.  Device-timed with
    CUDA events; inputs are 3 GB, far larger than L2."""
    import torch
    import stipple_b200 as sb
    from stipple_b200 import synth
    W, H = HEADLINE["width"], HEADLINE["height"]
    n = a.block_clip
    clip = synth.video_clip_device(W, H, 3, n)
    outs = torch.empty((n, H, W), dtype=torch.uint8, device="cuda")
    jobs = [dict(pixels=clip[f].data_ptr(), width=W, height=H, layout=sb.RGB8, palette_id=pid,
                 indices=outs[f].data_ptr()) for f in range(n)]
    res = {"workload": f"{n} frames of 3840x2160 RGB8 video, fixed 256-colour palette, "
                       "every frame in one call",
           "algorithmic_bytes_per_px": ALG_BYTES_PER_PX}
    px = n * W * H
    for B in (int(b) for b in a.block_sweep.split(",")):
        # The launch-shape tuner measures its candidates on the first calls.
        for _ in range(6):
            ctx.dither("blocks", jobs, stream=s, block=B)
        ctx.synchronize(s)
        ms_all = []
        for _ in range(2):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(torch.cuda.current_stream())
            ctx.dither("blocks", jobs, stream=s, block=B)
            e1.record(torch.cuda.current_stream())
            ctx.synchronize(s)
            ms_all.append(e0.elapsed_time(e1))
        ms = min(ms_all)
        gbs = px * ALG_BYTES_PER_PX / (ms / 1e3) / 1e9
        k = ctx.stats()
        res[f"B{B}"] = {"ms": ms, "mpx_s": px / ms / 1e3, "gb_s": gbs, "hbm_frac": gbs / hbm,
                        "launch": f"{k['block_threads']} threads x {k['block_min_ctas']} CTAs/SM"}
    del clip, outs, jobs
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
    src = synth.video_clip_device(W, H, 3, n).cpu().numpy()
    yuv = np.stack([synth.yuv444_frame(src[f]).reshape(-1) for f in range(n)])
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
        rgbaf[f].numpy().view(np.float32)[:] = synth.to_q16(src[f]).reshape(-1)
    res["e2e_rgbaf"] = e2e(rgbaf, sb.RGBAF32, sb.RGBAF32)
    return res


def bench_batched(ctx, s, a):
    import torch
    import stipple_b200 as sb
    from stipple_b200 import synth
    if a.batch == 512:
        spec, imgs = mixed_batch_images()
    else:
        spec = synth.mixed_batch_spec(a.batch)
        imgs = [synth.gradient_rgba8(w, h, seed) for w, h, seed, _ in spec]
    sizes = [(w, h) for w, h, _, _ in spec]
    jobs, keep, pids = [], [], []
    for (w, h, seed, colors), img in zip(spec, imgs):
        pid = ctx.palette_from_image(img, colors, associate_alpha=True)
        d = torch.from_numpy(img).cuda()
        o = torch.empty((h, w), dtype=torch.uint8, device="cuda")
        keep += [d, o]
        pids.append(pid)
        jobs.append(dict(pixels=d.data_ptr(), width=w, height=h, layout=sb.RGBA8, palette_id=pid,
                         indices=o.data_ptr()))
    total = sum(w * h for w, h in sizes)
    biggest = max(w * h for w, h in sizes)
    # Cold: the first call on these freshly made palettes (their uniform-key
    # tables are classified during it, and the segment-length tuner's first
    # call for this workload size runs untimed inside it).
    ctx.synchronize(s)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(torch.cuda.current_stream())
    ctx.dither("seq", jobs, stream=s)
    e1.record(torch.cuda.current_stream())
    ctx.synchronize(s)
    ms_cold = e0.elapsed_time(e1)
    for _ in range(max(WARM_CALLS, a.warmup)):  # the segment-length autotuner explores here
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
            "cold_batched_ms": ms_cold, "cold_batched_mpx_s": total / ms_cold / 1e3,
            "plain_ms": ms_p, "plain_mpx_s": total / ms_p / 1e3,
            "speedup": ms_p / ms_b, "amdahl_cap": total / biggest}


def serve_requests(n: int, seed: int):
    """The served mixed stream's requests: W and H log-uniform in 64..4096, RGB8
    or RGBA8 (half each, alpha-associated palettes for RGBA), colours from
    {2, 4, ..., 256}, engines 60 % sequential / 30 % block / 10 % Jacobi.  Each
    image is a crop of one of two seeded 4096x4096 frames at a random offset,
    submitted in place (no copy).  Returns (requests, base frames)."""
    from stipple_b200 import synth
    rng = np.random.default_rng(seed)
    sizes = synth.log_uniform_sizes(n, seed=seed + 1, lo=64, hi=4096)
    if "serve_base" not in _CACHE:
        _CACHE["serve_base"] = {False: synth.gradient_rgb8(4096, 4096, 3000),
                                True: synth.gradient_rgba8(4096, 4096, 3001)}
    base = _CACHE["serve_base"]
    reqs = []
    for w, h in sizes:
        alpha = bool(rng.random() < 0.5)
        y0 = int(rng.integers(0, 4096 - h + 1))
        x0 = int(rng.integers(0, 4096 - w + 1))
        colors = int(rng.choice([2, 4, 8, 16, 32, 64, 128, 256]))
        u = rng.random()
        engine = "seq" if u < 0.6 else ("blocks" if u < 0.9 else "jacobi")
        reqs.append((base[alpha][y0:y0 + h, x0:x0 + w], colors, engine, alpha))
    return reqs, base


def serve_stream(srv, reqs, rate: float, seed: int):
    """Poisson arrivals at `rate` requests/s from this thread; a second thread
    waits for the results in submission order and frees them as they come."""
    import queue
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=len(reqs))
    q: queue.Queue = queue.Queue()
    errors = []

    def waiter():
        while True:
            t = q.get()
            if t is None:
                return
            try:
                srv.wait(t)
            except Exception as e:  # noqa: BLE001 -- reported below
                errors.append(repr(e))

    th = threading.Thread(target=waiter)
    th.start()
    t0 = time.perf_counter()
    due = t0
    for (img, colors, engine, alpha), g in zip(reqs, gaps):
        due += g
        now = time.perf_counter()
        if due > now:
            time.sleep(due - now)
        q.put(srv.submit(img, colors, engine, alpha=alpha))
    q.put(None)
    th.join()
    if errors:
        raise RuntimeError(f"{len(errors)} served requests failed: {errors[0]}")
    return time.perf_counter() - t0


def bench_serve(ctx, a):
    """Served mixed stream (serve_requests): one server (120 GB admission budget,
    4 device workers, builders sized from the CPUs this process may use),
    warmed up by a separate stream, then `serve_requests` requests at each
    Poisson rate and, when --serve-stream is set, that many at the last rate.
    Latency = submission to result in host memory, with per-stage
    percentiles.  Beside it, the plain form: requests one at a time, one call
    each, on one context (a sample of the stream)."""
    import stipple_b200 as sb
    n = a.serve_requests
    reqs, _base = serve_requests(max(n, a.serve_stream), seed=77)
    total_px = sum(r[0].shape[0] * r[0].shape[1] for r in reqs[:n])
    rates = [float(r) for r in a.serve_rates.split(",") if r]
    aff = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else None
    srv = sb.Server(budget=120 << 30, workers=4)
    out = {"requests_per_rate": n, "total_px_per_rate": total_px,
           "workload": "served mixed stream: sizes log-uniform 64..4096, RGB/RGBA8, 2..256 "
                       "colours, 60/30/10 seq/block/Jacobi, Poisson arrivals, 120 GB admission",
           "cpu_count": os.cpu_count(), "affinity_cpus": aff}
    try:
        warm, _ = serve_requests(96, seed=4242)
        serve_stream(srv, warm, 2000.0, seed=1)
        st = srv.stats()
        out["host_threads"] = st["host_threads"]
        out["workers"] = st["workers"]
        for k, rate in enumerate(rates):
            srv.reset_stats()
            wall = serve_stream(srv, reqs[:n], rate, seed=100 + k)
            st = srv.stats()
            out[f"rate_{rate:g}"] = {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                                     "max_ms": st["max_ms"], "mpx_s": st["mpx_per_s"],
                                     "offered_mpx_s": total_px * rate / n / 1e6,
                                     "batches": st["batches"], "wall_s": wall,
                                     "completed": st["completed"], "stages": st["stages"],
                                     "peak_admitted_gb": st["peak_admitted_bytes"] / 2**30}
        if a.serve_stream > 0 and rates:
            srv.reset_stats()
            m = a.serve_stream
            wall = serve_stream(srv, reqs[:m], rates[-1], seed=999)
            st = srv.stats()
            out["stream"] = {"requests": m, "rate": rates[-1],
                             "total_px": sum(r[0].shape[0] * r[0].shape[1] for r in reqs[:m]),
                             "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "max_ms": st["max_ms"],
                             "mpx_s": st["mpx_per_s"], "batches": st["batches"], "wall_s": wall,
                             "completed": st["completed"], "stages": st["stages"],
                             "peak_admitted_gb": st["peak_admitted_bytes"] / 2**30}
    finally:
        srv.close()
    # Plain per-request form on a sample of the same requests.
    sample = reqs[:min(n, a.serve_plain)]
    lat = []
    t0 = time.perf_counter()
    for img, colors, engine, alpha in sample:
        t1 = time.perf_counter()
        tr = sb.Octree(np.ascontiguousarray(img), colors, alpha)
        pid = ctx.palette_from_octree(tr)
        ctx.dither_host(engine, img, pid)
        ctx.release_palette(pid)
        lat.append((time.perf_counter() - t1) * 1e3)
    plain_s = time.perf_counter() - t0
    px = sum(r[0].shape[0] * r[0].shape[1] for r in sample)
    out["plain"] = {"requests": len(sample), "mpx_s": px / plain_s / 1e6,
                    "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                    "wall_s": plain_s, "note": "service time per request, one at a time, no queueing"}
    return out


# ---------------------------------------------------------------- reference arm
def run_reference(a):
    from stipple_b200 import synth
    W, H, C = HEADLINE["width"], HEADLINE["height"], HEADLINE["colors"]
    img = synth.gradient_rgb8(W, H, HEADLINE["seed"])
    for _ in range(max(1, min(a.warmup, 1))):
        reference_cpu(img, C, budget_s=0.0)
    step_times = []
    cpu = {}
    for _ in range(max(1, a.steps)):
        cpu, t = reference_cpu(img, C, budget_s=0.0)
        step_times.extend(t)
    ms = statistics.median(step_times) * 1e3
    value = W * H / ms / 1e3
    # The baseline record describes the timed steps themselves.
    q1, q3 = (float(v) for v in np.percentile(step_times, [25, 75]))
    cpu.update({"value": value, "iqr_mpx_s": [W * H / q3 / 1e6, W * H / q1 / 1e6],
                "runs": len(step_times),
                "sample": f"{len(step_times)} sequential walks of the {W}x{H} frame ({C} colours), "
                          "median, palette build excluded; the walk is one dependent chain, so "
                          "one thread"})
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
        keep, jobs = [], []
        for w, h, seed, colors in synth.mixed_batch_spec(a.batch):
            im = synth.gradient_rgba8(w, h, seed)
            p = ctx.palette_from_image(im, colors, associate_alpha=True)
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
        opts = ({"seq_mode": a.seq_mode, "loop_mode": a.loop_mode, "walk_form": a.walk_form,
                 "seg_len": a.seg_len} if a.profile_case != "jacobi" else {})
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
