#!/usr/bin/env python
"""Benchmark: Msamples/s of the wavefront path tracer on one workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload large]

A step is one full frame: every pixel of the workload traced to its sample
count. The default workload is the large scene (1920x1080 at 64 spp, 16
bounces: a 2.09 M-triangle textured terrain, 500 glass/coat/fuzz instances,
4,096 lognormal emitters), the largest single-GPU configuration; `chart`
(1280x720, 64 spp, 12 bounces: the material chart under a 2048x1024 HDRI sky)
and `cornell` (256x256, 16 spp) are the smaller ones, and
`corpus:{cornell-box,veach-mis,teapot-full}` render the reference's pbrt
corpus at its published resolutions (1024^2, 1280x720, 1280x720) for a
ms/spp figure beside its own. `value` is device-timed (CUDA events on the
library's stream around each step) with the scene resident in HBM; `e2e` is
the same frame through the public API with a host camera update in and the
resolved image out to pinned host memory every step. Multi-GPU (torchrun):
rank r renders samples r*spp .. (r+1)*spp-1 of every pixel and the films are
summed with one NCCL all-reduce per step (weak scaling). The reference arm
times the CPU oracle (the reference's Rust/Vulkan path cannot be built or run
here) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

WORKLOADS = {
    "chart": dict(scene="chart", width=1280, height=720, spp=64, max_bounces=12,
                  label="material chart 5x5 icospheres (32,004 tris) + 2048x1024 HDRI sun sky + quad light, "
                        "1280x720, 64 spp, 12 bounces"),
    "cornell": dict(scene="cornell", width=256, height=256, spp=16, max_bounces=8,
                    label="closed box (36 tris) + 0.5x0.5 emitter, 256x256, 16 spp, 8 bounces"),
    "large": dict(scene="large", width=1920, height=1080, spp=64, max_bounces=16,
                  label="fBm terrain 1024^2 grid (2.09 M tris, 64 tiles) + 500 glass/coat/fuzz instances (~2k tris "
                        "each) + 4,096 lognormal(0,2) emitter triangles + 128 BC1/BC5 1024^2 textures, "
                        "1920x1080, 64 spp, 16 bounces"),
}
# The reference's pbrt corpus (imported scenes stored in tests/golden) at the
# resolutions of its published steady-state ms/spp on an RTX 4070 Ti SUPER
# (README.md:76-78): cross-hardware context, not a like-for-like baseline.
CORPUS = {
    "cornell-box": ("cornell_box", 1024, 1024, 5.5),
    "veach-mis": ("veach_mis", 1280, 720, 2.6),
    "teapot-full": ("teapot_full", 1280, 720, 8.0),
}
for _name, (_fx, _w, _h, _ms) in CORPUS.items():
    WORKLOADS[f"corpus:{_name}"] = dict(scene=f"corpus:{_fx}", width=_w, height=_h, spp=64, max_bounces=0,
                                        label=f"pbrt corpus {_name} (imported), {_w}x{_h}, 64 spp, the scene's "
                                              "max depth", reference_ms_per_spp=_ms)


BVH_BUILDERS = {"auto": 3, "host": 0, "gpu": 2, "gpu-ploc": 1}  # cenote_c.h CENOTE_BVH_*
BVH_LABELS = {0: "host SAH (sweep below 65,536 triangles), cost-optimal collapse",
              1: "GPU PLOC, cost-optimal collapse", 2: "GPU binned SAH, cost-optimal collapse"}


def bvh_builder(name):
    return BVH_BUILDERS[name]


def make_spec(w):
    """The workload's scene. Corpus scenes come from the committed fixtures;
    their max depth (pbrt's maxdepth) replaces the workload's 0."""
    from cenote_b200 import scenes
    if w["scene"].startswith("corpus:"):
        spec, extra = scenes.load_spec(ROOT / "tests" / "golden" / f"corpus_{w['scene'][7:]}.npz")
        if "sky_octahedral" in extra:
            from cenote_b200.pbrt import sky_environment
            spec.environment = sky_environment(extra["sky_octahedral"].astype(np.float32),
                                               extra["sky_world_from_light"], float(extra["sky_scale"]))
        w["max_bounces"] = spec.max_bounces
        return spec
    return {"chart": scenes.chart, "cornell": scenes.cornell, "large": scenes.large}[w["scene"]]()


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def l2_copy_peak(torch, mb=24, reps=100, trials=5):
    """Measured L2 bandwidth: `reps` device copies between two `mb`-MB
    buffers (48 MB together: L2-resident once warm) replayed as one CUDA
    graph, so launch gaps do not count; read + write bytes over CUDA-event
    time, best of `trials`."""
    a = torch.empty(mb << 20, dtype=torch.uint8, device="cuda")
    b = torch.empty_like(a)
    a.fill_(1)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        for _ in range(3):
            b.copy_(a)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(reps):
            b.copy_(a)
    g.replay()
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(trials):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * (mb << 20) * reps / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del g
    return best


def committed_traffic(workload):
    """Per-launch DRAM bytes of the traversal kernel from the committed ncu summary."""
    p = ROOT / "profiles" / f"traffic_{workload}.json"
    if p.exists():
        return json.loads(p.read_text())
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
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
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def rank_sample_range(rank: int, spp: int) -> tuple[int, int]:
    """The sample indices one rank renders for a multi-GPU frame: rank r takes
    [r * spp, (r + 1) * spp), so N ranks summing their films make one frame
    of N * spp distinct samples per pixel (weak scaling: spp per GPU)."""
    return rank * spp, spp


def cpu_baseline(spec, w, seconds=12.0):
    """The CPU oracle on all host cores, full-resolution frames at 1 spp until
    about `seconds` of work."""
    import oracle
    scene = oracle.OracleScene(spec)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    scene.render_sum(w["width"], w["height"], 0, 1, w["max_bounces"], threads=threads)
    one = time.perf_counter() - t0
    n = max(1, min(w["spp"], int(seconds / max(one, 1e-3))))
    t0 = time.perf_counter()
    scene.render_sum(w["width"], w["height"], 1, n, w["max_bounces"], threads=threads)
    dt = time.perf_counter() - t0
    samples = w["width"] * w["height"] * n
    return {"value": samples / dt / 1e6, "unit": "Msamples/s", "cores": threads, "kind": "port",
            "sample": f"{n} spp of the full {w['width']}x{w['height']} frame ({samples} samples, {dt:.1f} s)"}


def run_reference(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    spec = make_spec(w)
    scene = oracle.OracleScene(spec)
    threads = os.cpu_count() or 1
    # Each step: a bounded sample of the frame — 1 spp of every pixel.
    for k in range(args.warmup):
        scene.render_sum(w["width"], w["height"], k, 1, w["max_bounces"], threads=threads)
    t0 = time.perf_counter()
    for k in range(args.steps):
        scene.render_sum(w["width"], w["height"], args.warmup + k, 1, w["max_bounces"], threads=threads)
    dt = time.perf_counter() - t0
    value = w["width"] * w["height"] * args.steps / dt / 1e6
    line = {
        "impl": "reference", "metric": "Msamples/s", "value": value, "unit": "Msamples/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": w["label"], "width": w["width"], "height": w["height"], "spp": w["spp"],
                   "max_bounces": w["max_bounces"], "step": "1 spp of the full frame per step"},
        "cpu_baseline": {"value": value, "unit": "Msamples/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} x 1 spp of the full frame"},
        "e2e": {"value": value, "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's Rust/Vulkan renderer cannot be built (no cargo/slangc) or run (no Vulkan device) "
                "here; this arm is the CPU restatement of its kernels (oracle/), all host threads",
    }
    print(json.dumps(line), flush=True)


def run_guiding(args):
    """Learned guiding on the large scene: device time for plain and guided
    sampling to reach relMSE <= 0.01 against a plain render of
    `--reference-spp` samples, accumulating 4 spp at a time (the guide trains
    online from a seeded random initialisation, one Adam step of 65,536
    records after every 4-spp wave over the first 256 spp, then stays
    frozen)."""
    from cenote_b200 import Context, Film, Guide, Renderer, Scene, scenes
    from cenote_b200.metrics import rel_mse
    if int(os.environ.get("RANK", "0")) != 0:
        return
    W, H = args.width, args.height
    B = 16 if args.scene == "large" else 8
    ctx = Context(0)
    spec = scenes.SCENES[args.scene](W, H, 64, B)
    scene = Scene(ctx, spec)
    ref_r = Renderer(ctx, B)
    ref_f = Film(ctx, W, H)
    t0 = time.perf_counter()
    done = 0
    # The reference draws sample indices from 2^24 on, so it shares no samples
    # with the renders it judges.
    while done < args.reference_spp:
        n = min(512, args.reference_spp - done)
        ref_r.accumulate_range(scene, ref_f, (1 << 24) + done, n)
        done += n
    ref_s = time.perf_counter() - t0
    ref = ref_f.averages()[..., :3]
    target, chunk, cap = 0.01, 4, 4096

    def run(guided):
        r = Renderer(ctx, B, samples_per_wave=chunk)
        g = None
        if guided:
            g = Guide(ctx, seed=11)
            r.set_guide(g, 0.5, 1, 5e-3)
        f = Film(ctx, W, H)
        ms, spp, err, curve = 0.0, 0, float("inf"), []
        while spp < cap:
            if guided and spp == 256:
                r.set_guide(g, 0.5, 0, 5e-3)  # the guide trained long enough: freeze it
            r.accumulate(scene, f, chunk)
            ms += r.stats()["gpu_ms"]
            spp += chunk
            err = rel_mse(f.averages()[..., :3], ref)
            if spp in (16, 64, 256, 1024) or err <= target:
                curve.append({"spp": spp, "ms": round(ms, 2), "rel_mse": err})
            if err <= target:
                break
        return {"ms": ms, "spp": spp, "rel_mse": err, "reached": err <= target, "curve": curve}

    plain = run(False)
    guided = run(True)
    line = {
        "metric": "device time to relMSE <= 0.01, guided / plain", "value": guided["ms"] / plain["ms"],
        "unit": "ratio", "higher_is_better": False, "n_gpus": 1, "scaling": "none", "vs_baseline": None,
        "dtype": "f32 (guide MLP bf16 with f32 accumulation)", "data": "synthetic (procedural scene, seeded)",
        "config": {"workload": f"{args.scene} at {W}x{H}, {B} bounces, reference {args.reference_spp} spp plain; "
                               "4-spp chunks; guide: 8 vMF lobes, 3x64 hidden, one-sample MIS weight 0.5, "
                               "1 Adam step (lr 5e-3, batch 65,536) per wave for the first 256 spp, then frozen"},
        "plain": plain, "guided": guided, "reference_s": ref_s,
    }
    print(json.dumps(line), flush=True)


def run_serving(args):
    """The batched-serving workload: a seeded Poisson stream (200 jobs/s) of
    progressive render jobs drawn uniformly from the closed box, the material
    chart and the large scene, at a resolution uniform in {256², 640x360,
    1280x720, 1920x1080} and a target spp log-uniform in 1..256, admitted
    against a 160 GB budget with a frame every 4 spp. With --concurrency C
    the same job draws run as a closed loop instead: C jobs in flight, each
    completion submitting the next. Reports time to first frame and time to
    target spp (p50/p99 over jobs, submission to event, on the server's clock)
    and the aggregate samples/s from the first submission to the last
    completion."""
    from cenote_b200 import JOB_DONE, JOB_FAILED, Context, Scene, Server, scenes
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ctx = Context(0)
    specs = {"box": (scenes.cornell, 8), "chart": (scenes.chart, 12), "large": (scenes.large, 16)}
    resident = {k: Scene(ctx, f()) for k, (f, _) in specs.items()}
    rng = np.random.default_rng(3)
    res = [(256, 256), (640, 360), (1280, 720), (1920, 1080)]
    names = list(specs)
    arrivals = np.cumsum(rng.exponential(1.0 / 200.0, args.jobs))
    jobs = []
    for k in range(args.jobs):
        n = names[rng.integers(3)]
        w, h = res[rng.integers(4)]
        spp = int(np.clip(np.rint(np.exp(rng.uniform(0.0, np.log(256.0)))), 1, 256))
        jobs.append((float(arrivals[k]), n, w, h, spp))
    server = Server(ctx, 160 << 30, slots=args.slots, frame_spp=4, max_active=64)
    # One small job per scene first: graph instantiation and first-touch costs
    # stay out of the measured stream; then 32 one-sample jobs per resolution,
    # whose film and frame buffers the server keeps for reuse, so the stream
    # does not measure first-time allocations either.
    for n in names:
        server.wait(server.submit(resident[n], 64, 64, 4, specs[n][1]))
    warm = [server.submit(resident["box"], w, h, 1, 1) for w, h in res for _ in range(32)]
    for j in warm:
        server.wait(j)
    ids = []
    done = {}  # job -> its status when it finished; finished jobs are released at once
    live = []

    def harvest():
        nonlocal live
        keep = []
        for j in live:
            s_ = server.poll(j)
            if s_.state in (JOB_DONE, JOB_FAILED):
                done[j] = s_
                server.release(j)  # a finished job's host-side result is not kept
            else:
                keep.append(j)
        live = keep

    with ClockSampler(0) as clocks:
        t0 = time.perf_counter()
        if args.concurrency:
            # Closed loop: `concurrency` jobs in flight, each completion
            # submitting the stream's next job at once.
            pending = list(jobs)
            while pending or live:
                while pending and len(live) < args.concurrency:
                    _, n, w, h, spp = pending.pop(0)
                    j = server.submit(resident[n], w, h, spp, specs[n][1])
                    ids.append(j)
                    live.append(j)
                time.sleep(0.002)  # each poll takes the server's lock: keep the loop light
                harvest()
        else:
            last = 0.0
            for at, n, w, h, spp in jobs:
                while True:
                    now = time.perf_counter() - t0
                    if now >= at:
                        break
                    if now - last > 0.25 and at - now > 0.005:  # a poll per live job: keep it rare
                        harvest()
                        last = time.perf_counter() - t0
                    else:
                        time.sleep(min(at - now, 0.002))
                j = server.submit(resident[n], w, h, spp, specs[n][1])
                ids.append(j)
                live.append(j)
        deadline = time.perf_counter() + 1800.0
        while live and time.perf_counter() < deadline:
            harvest()
            time.sleep(0.05)
    counters = server.stats()
    st = [done[j] if j in done else server.poll(j) for j in ids]
    ttff = np.array([s.first_frame_ms - s.submit_ms for s in st])
    burst_end = max(s.first_frame_ms for s in st[:args.concurrency]) if args.concurrency else 0.0
    ttt = np.array([s.done_ms - s.submit_ms for s in st])
    span_ms = max(s.done_ms for s in st) - min(s.submit_ms for s in st)
    samples = sum(w * h * spp for _, _, w, h, spp in jobs)
    pct = lambda a, q: float(np.percentile(a, q))
    line = {
        "metric": "p99 time to first frame (batched serving)", "value": pct(ttff, 99), "unit": "ms",
        "higher_is_better": False, "n_gpus": 1, "scaling": "none", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (procedural scenes, seeded job stream)",
        "config": {"workload": (f"{args.jobs} jobs, closed loop with {args.concurrency} jobs in flight"
                                if args.concurrency else f"{args.jobs} jobs, Poisson 200/s")
                               + ", scenes {closed box, material chart, large}, "
                               "resolutions {256^2, 640x360, 1280x720, 1920x1080}, spp log-uniform 1..256, "
                               f"160 GB budget, job-tagged waves on {args.slots} lane(s) (16 M-path pool each, "
                               "first-frame waves on high-priority streams), 64 resident jobs, a frame every 4 spp"},
        "time_to_first_frame_ms": {"p50": pct(ttff, 50), "p99": pct(ttff, 99), "max": float(ttff.max())},
        "time_to_target_ms": {"p50": pct(ttt, 50), "p99": pct(ttt, 99), "max": float(ttt.max())},
        # Closed loop: the jobs after the first `concurrency`, which all arrive
        # at once when the loop starts; and those submitted once the opening
        # burst's last first frame is out (past its transient).
        "steady_state_time_to_first_frame_ms": (
            {"p50": pct(ttff[args.concurrency:], 50), "p99": pct(ttff[args.concurrency:], 99),
             "jobs": int(len(ttff) - args.concurrency)} if args.concurrency and len(ttff) > args.concurrency else None),
        "after_opening_burst_time_to_first_frame_ms": (
            (lambda sel: {"p50": pct(ttff[sel], 50), "p99": pct(ttff[sel], 99), "max": float(ttff[sel].max()),
                          "jobs": int(sel.sum()), "burst_cleared_ms": burst_end})(
                np.array([s.submit_ms > burst_end for s in st]))
            if args.concurrency and any(s.submit_ms > burst_end for s in st) else None),
        "slowest_first_frames": [
            {"job": int(k), "scene": jobs[k][1], "size": f"{jobs[k][2]}x{jobs[k][3]}", "spp": jobs[k][4],
             "submit_ms": round(st[k].submit_ms, 1), "ttff_ms": round(float(ttff[k]), 1)}
            for k in np.argsort(-ttff)[:6]],
        "aggregate_msamples_per_s": samples / (span_ms / 1e3) / 1e6,
        "samples": samples, "span_ms": span_ms,
        "failed": int(sum(1 for s in st if s.state != JOB_DONE)),
        "waves": {"count": counters["waves"], "first_frame_waves": counters["first_waves"],
                  "mean_paths": counters["wave_paths"] / max(1, counters["waves"]),
                  "device_busy_ms": counters["busy_ms"], "wall_ms": counters["wall_ms"]},
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)
    server.close()


def run_knob_sweep(args, w):
    """The launch knobs one at a time around the autotuner's choice: device
    ms per sample of every pixel (the better of 3 runs of 16 spp) for each
    value of each knob, the others held at the tuned setting. One JSON line."""
    from cenote_b200 import Context, Film, Renderer, Scene

    ctx = Context(0)
    ctx.set_bvh_builder(bvh_builder(args.bvh))
    scene = Scene(ctx, make_spec(w))
    W, H = w["width"], w["height"]
    r = Renderer(ctx, w["max_bounces"])
    t0 = time.perf_counter()
    best = r.autotune(scene, W, H)
    tune_s = time.perf_counter() - t0
    film = Film(ctx, W, H)
    spp = 16

    def timed(knobs):
        r.set_tuning(*knobs)
        ms = []
        for _ in range(3):
            r.accumulate(scene, film, spp)
            ms.append(r.stats()["gpu_ms"])
        return round(min(ms) / spp, 4)

    names = ("material_sort", "samples_per_wave", "refill_idle", "top_nodes", "l2_window", "per_lane_triangles",
             "block_size", "stack_depth", "sort_by_location")
    base = tuple(best[k] for k in names)
    values = ((0, 1, 2), (0, 4, 8, 16), (4, 8, 16, 32), (0, 80, 320), (0, 1), (0, 1), (128, 256), (16, 32), (0, 1))
    sweep = {"tuned": timed(base)}
    for i, vals in enumerate(values):
        for v in vals:
            k = list(base)
            k[i] = v
            sweep[f"{names[i]}={v}"] = timed(tuple(k))
    line = {"metric": "device ms per sample of every pixel, one knob varied", "unit": "ms", "workload": w["label"],
            "autotuned": {k: best[k] for k in names}, "autotune_s": round(tune_s, 2),
            "samples_per_call": spp, "note": "samples_per_wave above 16 equals 16 at 16 spp per call",
            "sweep": sweep}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large", choices=list(WORKLOADS) + ["serving", "guiding"])
    ap.add_argument("--jobs", type=int, default=256, help="serving: jobs in the Poisson stream")
    ap.add_argument("--slots", type=int, default=2, help="serving: lanes (path pool + stream pair each), 1 or 2")
    ap.add_argument("--concurrency", type=int, default=0,
                    help="serving: keep this many jobs in flight (closed loop) instead of the Poisson arrivals")
    ap.add_argument("--width", type=int, default=480, help="guiding: image width")
    ap.add_argument("--height", type=int, default=270, help="guiding: image height")
    ap.add_argument("--reference-spp", type=int, default=16384, help="guiding: spp of the plain reference")
    ap.add_argument("--scene", default="large", choices=["large", "ceiling_box"], help="guiding: the scene")
    ap.add_argument("--spp", type=int, default=0, help="override the workload's spp (profiling runs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--bvh", default="auto", choices=list(BVH_BUILDERS),
                    help="BVH builder (scene prep, outside the timed region): auto = GPU binned SAH from 2^20 "
                         "triangles, else host SAH; host; gpu (binned SAH); gpu-ploc")
    ap.add_argument("--tuning", default="",
                    help="pin the launch knobs instead of autotuning: sort,samples_per_wave,refill,top_nodes,l2"
                         "[,per_lane_triangles[,block_size,stack_depth[,sort_by_location]]] "
                         "(profiling runs that must not record the tuner's probes)")
    ap.add_argument("--material-sort", type=int, default=None, choices=[0, 1, 2],
                    help="fix the material sort (0 off, 1 every bounce, 2 from the first bounce on) "
                         "instead of autotuning the launch knobs")
    ap.add_argument("--sweep-knobs", action="store_true",
                    help="instead of the bench: time each launch knob around the autotuned setting")
    args = ap.parse_args()
    if args.workload == "serving":
        run_serving(args)
        return
    if args.workload == "guiding":
        run_guiding(args)
        return
    w = dict(WORKLOADS[args.workload])
    if args.spp:
        w["spp"] = args.spp
    if args.sweep_knobs:
        run_knob_sweep(args, w)
        return
    if args.impl == "reference":
        run_reference(args, w)
        return

    import torch
    import torch.distributed as dist
    from cenote_b200 import PROFILE_COUNTS, PROFILE_TIMING, Context, Film, Renderer, Scene, scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    spec = make_spec(w)
    W, H, spp, maxb = w["width"], w["height"], w["spp"], w["max_bounces"]
    ctx = Context(local)
    ctx.set_bvh_builder(bvh_builder(args.bvh))
    t0 = time.perf_counter()
    scene = Scene(ctx, spec)
    prep_wall_ms = (time.perf_counter() - t0) * 1e3
    prep = scene.prep_times_ms()
    r = Renderer(ctx, maxb)
    t_tune = time.perf_counter()
    if args.tuning:
        r.set_tuning(*[int(x) for x in args.tuning.split(",")])
        tuning = r.tuning()
    elif args.material_sort is None:
        tuning = r.autotune(scene, W, H)  # per-scene launch knobs, outside the timed region
    else:
        r.set_tuning(args.material_sort)
        tuning = r.tuning()
    tune_s = time.perf_counter() - t_tune
    film = Film(ctx, W, H)
    stream = torch.cuda.ExternalStream(ctx.stream)

    # Traversal visit counts for the roofline's algorithmic bytes: one
    # instrumented frame, outside the timed region.
    r.set_profiling(PROFILE_COUNTS)
    film.reset()
    r.accumulate(scene, film, spp)
    counts = r.stats()
    r.set_profiling(PROFILE_TIMING)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > L2 (126 MB)
    sum_view = None
    if world > 1:
        class _Dev:
            def __init__(self, ptr, n):
                self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 2}
        sum_view = torch.as_tensor(_Dev(film.device_sums(), W * H * 4), device="cuda")

    first_sample, _ = rank_sample_range(rank, spp)

    def step(k):
        film.reset()
        r.accumulate_range(scene, film, first_sample, spp)  # synchronous: returns when the frame is done
        if sum_view is not None:
            dist.all_reduce(sum_view)  # the frame's N * spp samples per pixel
            torch.cuda.synchronize()

    for k in range(args.warmup):
        step(k)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    stage = {"intersect_ms": 0.0, "shade_ms": 0.0, "shadow_ms": 0.0, "raygen_ms": 0.0, "film_ms": 0.0}
    launches = 0
    rays = [0, 0]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                evs[k][0].record(stream)
            step(k)
            evs[k][1].record(stream)
            st = r.stats()
            for key in stage:
                stage[key] += st[key]
            launches += st["kernel_launches"]
            rays[0] += st["extension_rays"]
            rays[1] += st["shadow_rays"]
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    samples_total = W * H * spp * args.steps * world
    value = samples_total / (ms / 1e3) / 1e6

    # e2e through the public API: camera in from the host, image out to pinned host memory.
    r.set_profiling(0)
    pinned = torch.empty((H, W, 4), dtype=torch.float32, pin_memory=True)
    e2e_ms = []
    for k in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t_a = time.perf_counter()
        scene.set_camera(spec.camera)
        film.reset()
        r.accumulate_range(scene, film, first_sample, spp)
        if sum_view is not None:
            dist.all_reduce(sum_view)  # the frame's sums, read back whole (N * spp samples per pixel)
            pinned.view(-1).copy_(sum_view)
        else:
            film.averages_into(pinned.data_ptr())
        t_b = time.perf_counter()
        if k >= args.warmup:
            e2e_ms.append((t_b - t_a) * 1e3)
    e2e_step = float(np.mean(e2e_ms))
    if world > 1:
        t = torch.tensor([e2e_step], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_step = float(t.item())
    e2e_value = W * H * spp * world / (e2e_step / 1e3) / 1e6

    # Roofline of the traversal kernels (intersect + shadow): the
    # algorithmic bytes per ray = 32 (origin, direction) + 4 (queue slot) +
    # 16 (hit record) for extension rays or 64 (shadow record) for shadow
    # rays, plus 80 B per wide node visited and 36 B per triangle tested.
    ext, shd = counts["extension_rays"], counts["shadow_rays"]
    alg_bytes_frame = ext * (32 + 4 + 16) + shd * 64 + 80 * counts["node_visits"] + 36 * counts["triangle_tests"]
    trav_ms_frame = (stage["intersect_ms"] + stage["shadow_ms"]) / args.steps
    trav_launches = 2 * maxb * counts["waves"]
    achieved = alg_bytes_frame / (trav_ms_frame / 1e3) / 1e9 if trav_ms_frame > 0 else None
    peak, peak_kind = measured_peaks()
    l2_peak = l2_copy_peak(torch)
    traffic = committed_traffic(args.workload)
    # DRAM bytes per traversal launch from the committed capture of a smaller
    # wave, scaled by paths per wave (a first-order model: the per-ray
    # path-state traffic grows with the rays per launch).
    wave_paths = W * H * min(counts["samples_per_wave"], spp)
    traffic_per_launch = (traffic["bytes_per_launch_captured"] * wave_paths / traffic["captured_paths_per_wave"]
                          if traffic and "captured_paths_per_wave" in traffic else None)
    # Shading: bytes per path vertex = 72 path in + 52 path out + 128
    # geometry record + 144 material + 12 indices + 96 vertex attributes +
    # 64 shadow record + 16 radiance read-modify-write = 584 for a surface
    # hit; a miss reads its path (72) and adds its radiance (16) = 88.
    hits = counts["surface_hits"]
    shade_bytes_frame = 584 * hits + 88 * (ext - hits)
    shade_ms_frame = stage["shade_ms"] / args.steps
    shade_achieved = shade_bytes_frame / (shade_ms_frame / 1e3) / 1e9 if shade_ms_frame > 0 else None
    # The BVH and triangles of the chart and the closed box fit in L2 (the
    # L2 roofline bounds their walk); the large scene's do not (HBM).
    l2_resident = args.workload != "large"

    line = {
        "metric": "Msamples/s", "value": value, "unit": "Msamples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (procedural scene, seeded)",
        "config": {"workload": w["label"], "width": W, "height": H, "spp": spp, "max_bounces": maxb,
                   "parallelism": f"sample ranges x{world}, films summed by all-reduce" if world > 1 else "1 GPU",
                   "l2": "256 MB buffer written between timed steps (L2 flush); the path pool per wave also "
                         "exceeds L2",
                   "samples_per_wave": counts["samples_per_wave"], "waves_per_step": counts["waves"],
                   "tuning": {"material_sort": ["off", "every bounce", "secondary bounces"][tuning["material_sort"]],
                              "samples_per_wave": tuning["samples_per_wave"] or "automatic",
                              "refill_idle": tuning["refill_idle"] or 8,
                              "top_nodes_in_shared_memory": tuning["top_nodes"],
                              "l2_persisting_bvh": bool(tuning["l2_window"]),
                              "triangle_tests": "per lane" if tuning["per_lane_triangles"] else "warp queue",
                              "traversal_block_size": tuning["block_size"],
                              "traversal_stack_depth": tuning["stack_depth"],
                              "sort_key": "location" if tuning["sort_by_location"] else "instance",
                              "chosen_by": "autotuner" if args.material_sort is None and not args.tuning else "flag",
                              "autotune_s": round(tune_s, 3)},
                   "guides": "albedo, normal and depth traced and accumulated every sample, as Renderer::accumulate does"},
        "e2e": {"value": e2e_value, "unit": "Msamples/s", "ms_per_step": e2e_step,
                "h2d_bytes_per_step": 48, "d2h_bytes_per_step": W * H * 16},
        "gpu_launches": launches,
        "rays_per_s": (rays[0] + rays[1]) * world / (ms / 1e3),
        "extension_rays_per_step": rays[0] / args.steps, "shadow_rays_per_step": rays[1] / args.steps,
        "stage_ms_per_step": {k: v / args.steps for k, v in stage.items()},
        "scene_prep_ms": {"bvh": float(prep[0]), "bvh_builder": BVH_LABELS[scene.bvh_builder()],
                          "env_tables": float(prep[1]), "total": float(prep[2]), "wall": prep_wall_ms},
        "roofline": {
            "kernel": "traversal (k_intersect + k_shadow)", "bound": "hbm",
            "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
            "traffic": traffic_per_launch,
            "algorithmic_bytes_per_launch": alg_bytes_frame / max(1, trav_launches),
            "launch_ms": trav_ms_frame / max(1, trav_launches),
            "nodes_per_ray": counts["node_visits"] / max(1, ext + shd),
            "tris_per_ray": counts["triangle_tests"] / max(1, ext + shd),
            "applies": "HBM roofline: the BVH exceeds L2" if not l2_resident else
                       "the BVH is L2-resident: roofline_l2 is the bound that applies",
        },
        "roofline_l2": {
            "kernel": "traversal (k_intersect + k_shadow)", "bound": "l2", "achieved": achieved, "peak": l2_peak,
            "unit": "GB/s", "frac": (achieved / l2_peak) if achieved else None,
            "peak_source": "measured in this run: 100 copies between two 24 MB buffers (L2-resident), one CUDA graph",
        },
        "roofline_shade": {
            "kernel": "k_shade", "bound": "hbm", "achieved": shade_achieved, "peak": peak, "unit": "GB/s",
            "frac": (shade_achieved / peak) if shade_achieved else None, "peak_source": peak_kind,
            "algorithmic_bytes_per_frame": shade_bytes_frame, "surface_hits_per_frame": hits,
            "misses_per_frame": ext - hits, "ms_per_frame": shade_ms_frame,
            "bytes_per_vertex": "584 per surface hit, 88 per miss",
        },
    }
    if "reference_ms_per_spp" in w:
        line["corpus"] = {"ms_per_spp": ms / args.steps / spp, "reference_ms_per_spp": w["reference_ms_per_spp"],
                          "reference_hardware": "RTX 4070 Ti SUPER, Vulkan ray query (README.md:76-78)",
                          "note": "cross-hardware context, not a baseline: the reference publishes only these"}
    if rank == 0:
        line["clocks"] = clocks.summary()
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(spec, w)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
