"""Benchmark of the plain GPU path tracer on the 1,048,576-triangle sphere-grid workload
(1920x1080, 64 spp, 16 bounces, 2048x1024 sky with a 5e4 sun disk).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

A step renders the whole workload once (132.7 M camera samples). `value` is Msamples/s with
the scene resident in HBM (CUDA-event time of the render's kernels, max over ranks); `e2e`
is the same metric through the C ABI with host buffers: scene upload, render and film
download every step. With --gpus N each rank renders its own replica (seed 42 + rank):
weak scaling, no collective on the data path. `--impl reference` times the reference's
own CPU renderer (built from its sources) on this host's cores instead.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cpu-renderer_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "Msamples/s"
UNIT = "Msamples/s"
WORKLOAD = "sphere-grid-1M-1920x1080-64spp-d16"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-spp", type=int, default=4)
    ap.add_argument("--workload", default="grid", choices=["grid", "batch", "serve", "guided"],
                    help="grid: the 1M-triangle 1080p render (default); batch: 64 uneven scenes in one pool "
                         "against one by one; serve: a Poisson request stream through the server")
    ap.add_argument("--requests", type=int, default=400, help="serve: requests in the stream (2000 for the full run)")
    ap.add_argument("--rate", type=float, default=40.0, help="serve: arrivals per second")
    ap.add_argument("--literal-clutter", action="store_true",
                    help="batch/serve: keep config 1's triangle sizes at every triangle count")
    ap.add_argument("--engine-iters", type=int, default=0,
                    help="serve: iterations between the engine's host checks (0: the engine's default)")
    ap.add_argument("--mix-scale", type=float, default=1.0,
                    help="batch/serve: scale every job's width and height (quick runs)")
    ap.add_argument("--solo-log2", type=int, default=0,
                    help="batch: jobs of at least 2^n samples render alone beside the pool (0: the library's 24; "
                         "64: every job shares the pool)")
    ap.add_argument("--frame", default="1920x1080",
                    help="guided: the learned-proposal scene's frame (the 1080p workload's frame by default)")
    return ap.parse_args()


from replicas import Replicas, dist_env  # noqa: E402  (after the package path is set)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
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
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def build_workload(spp):
    import crgpu
    import workloads
    sc = workloads.sphere_grid_scene(samples=spp)
    tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
    nodes, idx = crgpu.build_bvh(tris)
    return sc, tris, nodes, idx


def flush_l2(torch, device):
    buf = torch.empty(64 << 20, dtype=torch.float32, device=device)  # 256 MB > 126 MB L2
    buf.zero_()
    torch.cuda.synchronize(device)
    del buf


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return p.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def profile_summary():
    """The committed ncu summary of k_trace (DRAM bytes per traced ray, L2 throughput), or {}."""
    path = os.path.join(ROOT, "profiles", "k_trace_sphere_grid.json")
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def profile_traffic():
    """DRAM bytes per traced ray (closest or any hit) of k_trace from the committed ncu summary."""
    return profile_summary().get("dram_bytes_per_traced_ray")


def cpu_reference_rate(sc, spp, threads):
    """The reference's cr::render on this host's cores: Msamples/s on a bounded sample."""
    import refimpl
    if not refimpl.available():
        return None
    rs = refimpl.RefScene(sc["triangles"], sc["materials"]).build_bvh()
    env = refimpl.RefEnvironment(image=sc["env_image"])
    o = sc["options"]
    from cr_types import Options
    opt = Options.make(width=o.width, height=o.height, samples=spp, bounces=o.bounces, threads=threads, seed=o.seed)
    film, st = rs.render(sc["camera"], opt, env)
    return st["camera_samples"] / st["seconds"] / 1e6, st


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import refimpl
    if not refimpl.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref/libcr_ref.so was not built"}))
        return
    threads = os.cpu_count() or 1
    # the scene generator and the ctypes layouts only: the reference finalizes the scene and
    # builds its BVH itself, and the product library is never loaded on this arm
    import workloads
    from cr_types import Options
    sc = workloads.sphere_grid_scene(samples=args.spp)
    rs = refimpl.RefScene(sc["triangles"], sc["materials"]).build_bvh()
    env = refimpl.RefEnvironment(image=sc["env_image"])
    o = sc["options"]
    step_spp = 1  # one step: the full 1920x1080 frame at 1 spp of the same streams
    opt = Options.make(width=o.width, height=o.height, samples=step_spp, bounces=o.bounces, threads=threads, seed=o.seed)
    for _ in range(args.warmup):
        rs.render(sc["camera"], opt, env)
    secs = []
    for _ in range(args.steps):
        _, st = rs.render(sc["camera"], opt, env)
        secs.append(st["seconds"])
    samples = o.width * o.height * step_spp
    value = samples * len(secs) / sum(secs) / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded procedural scene and sky)",
        "config": {"workload": WORKLOAD, "triangles": 1 << 20, "width": o.width, "height": o.height, "spp": args.spp,
                   "bounces": o.bounces, "step": f"{o.width}x{o.height} x {step_spp} spp of the same sample streams",
                   "same_config": "same scene, frame, bounces and per-sample streams; a step is 1 of the 64 samples "
                                  "per pixel, so the per-sample rate is comparable and the step is 1/64 of the render"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{o.width}x{o.height} x {step_spp} spp per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_ours(args):
    _, _, local = dist_env()
    import torch
    import crgpu
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    ranks = Replicas("nccl", device)
    rank, world = ranks.rank, ranks.world
    sc, tris, nodes, idx = build_workload(args.spp)
    cam, opt = sc["camera"], sc["options"]
    opt.seed = ranks.seed(42)
    env = crgpu.env_desc(image=sc["env_image"])
    g = crgpu.GpuScene(tris, sc["materials"], env=env, bvh=(nodes, idx), device=local)
    samples_per_step = opt.width * opt.height * opt.samples
    barrier = ranks.barrier

    # counting pass (untimed): node pairs and triangles per closest-hit and any-hit ray
    tc = crgpu.Tuning()
    tc.count_traversal = 1
    copt = crgpu.Options.make(width=opt.width, height=opt.height, samples=1, bounces=opt.bounces, seed=opt.seed)
    cstats, _ = g.render_resident(cam, copt, tuning=tc)
    ext_pairs = cstats["extend_pairs"] / max(1, cstats["extend_rays"])
    ext_tris = cstats["extend_triangles"] / max(1, cstats["extend_rays"])
    sh_pairs = cstats["shadow_pairs"] / max(1, cstats["shadow_rays"])
    sh_tris = cstats["shadow_triangles"] / max(1, cstats["shadow_rays"])

    for _ in range(args.warmup):
        g.render_resident(cam, opt)
    # timed: device time of K renders; phase timing in a separate pass below
    dev_ms, launches, ext_rays = [], 0, 0
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush_l2(torch, device)
            barrier()
            st, _ = g.render_resident(cam, opt)
            barrier()
            dev_ms.append(st["device_ms"])
            launches += st["kernel_launches"]
    max_ms = ranks.max_over_ranks(sum(dev_ms))
    value = ranks.whole_job_rate(samples_per_step * args.steps, max_ms / 1e3)

    # the same renders with alias-table environment sampling (other sample streams, the same
    # unbiased estimator): K more timed steps after one untimed render that builds the table
    ta = crgpu.Tuning()
    ta.env_alias = 1
    g.render_resident(cam, opt, tuning=ta)
    alias_ms = []
    for _ in range(args.steps):
        flush_l2(torch, device)
        barrier()
        st, _ = g.render_resident(cam, opt, tuning=ta)
        barrier()
        alias_ms.append(st["device_ms"])
    alias_max = ranks.max_over_ranks(sum(alias_ms))
    alias_value = ranks.whole_job_rate(samples_per_step * args.steps, alias_max / 1e3)

    # dominant-kernel timing: one more render with CUDA events around every launch
    tp = crgpu.Tuning()
    tp.time_phases = 1
    pst, _ = g.render_resident(cam, opt, tuning=tp)
    trace_launches = pst["iterations"]
    # algorithmic bytes: 64 B per node pair, 48 B per triangle record, plus the ray's own
    # state (closest hit: ray 32 + flags/ignore/pixel/sample 16 + result 4; any hit: ray 48 +
    # contribution 16 + radiance read/write 32 + flags 4)
    ext_bytes = 64.0 * ext_pairs + 48.0 * ext_tris + 52.0
    sh_bytes = 64.0 * sh_pairs + 48.0 * sh_tris + 100.0
    algo_bytes = ext_bytes * pst["extend_rays"] + sh_bytes * pst["shadow_rays"]
    achieved = algo_bytes / (pst["trace_ms"] / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic_per_ray = profile_traffic()
    rays = pst["extend_rays"] + pst["shadow_rays"]
    roofline = {
        "kernel": "k_trace (closest + any hit)", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": achieved / peak, "peak_source": peak_kind,
        "traffic": (traffic_per_ray * rays / trace_launches) if traffic_per_ray else None,
        "l2": profile_summary().get("l2"),
        "algorithmic_bytes_per_launch": algo_bytes / trace_launches,
        "closest_hit": {"bytes_per_ray": ext_bytes, "pairs_per_ray": ext_pairs, "triangles_per_ray": ext_tris},
        "any_hit": {"bytes_per_ray": sh_bytes, "pairs_per_ray": sh_pairs, "triangles_per_ray": sh_tris},
        "trace_ms_share": pst["trace_ms"] / pst["device_ms"],
        "shade_ms_share": pst["shade_ms"] / pst["device_ms"],
        "mrays_per_s": rays / (pst["trace_ms"] / 1e3) / 1e6,
        "launches": trace_launches,
    }

    # end to end through the C ABI with host buffers: upload, render, download every step
    # (K steps, each a new scene handle: create + render + film download + destroy), after one
    # untimed step of the same kind (the first scene handle's device blocks are fresh
    # allocations; later ones reuse the blocks the previous handle freed)
    e2e_secs = []
    film = None
    for step in range(args.steps + 1):
        barrier()
        t0 = time.perf_counter()
        ge = crgpu.GpuScene(tris, sc["materials"], env=env, bvh=(nodes, idx), device=local)
        film, _ = ge.render(cam, opt)
        ge.close()
        barrier()
        if step:
            e2e_secs.append(time.perf_counter() - t0)
    e2e_value = ranks.whole_job_rate(samples_per_step * args.steps, sum(e2e_secs))
    h2d_bytes = int(tris.nbytes + nodes.nbytes + idx.nbytes + sc["env_image"].nbytes + sc["materials"].nbytes)
    d2h_bytes = int(film.nbytes)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        r = cpu_reference_rate(sc, args.cpu_sample_spp, threads)
        if r is not None:
            cpu = {"value": r[0], "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"{opt.width}x{opt.height} x {args.cpu_sample_spp} spp of the same scene and streams "
                             f"({r[1]['seconds']:.1f} s)"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic (seeded procedural scene and sky)",
            "config": {"workload": WORKLOAD, "triangles": int(len(tris)), "width": opt.width, "height": opt.height,
                       "spp": opt.samples, "bounces": opt.bounces, "env": "2048x1024 log-normal + 0.5 deg sun 5e4",
                       "parallelism": f"replicas x{world}", "l2": "256 MB buffer written between timed steps",
                       "traversal": "fp32 conservative boxes + fp64 reference triangle test"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes,
                    "step_seconds": [round(x, 4) for x in e2e_secs],
                    "note": "cr_gpu_scene_create (upload) + cr_gpu_render (film download) + destroy from host arrays, "
                            "every one of K steps, after one untimed step of the same kind"},
            "env_alias": {"value": alias_value, "unit": UNIT, "ms_per_step": alias_max / args.steps,
                          "note": "alias-table environment sampling instead of the reference's CDF search "
                                  "(different sample streams, exact realised texel densities); value above is "
                                  "the CDF (reference-stream) mode"},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
        }
        print(json.dumps(line))
    g.close()
    ranks.close()


def mix_scenes(env_size=None, literal=False):
    """The 64 uneven scenes of the multi-scene mix on the device: [(GpuScene, camera)]."""
    import crgpu
    import workloads
    out = []
    for i, (count, seed, _, _) in enumerate(workloads.uneven_scene_mix()):
        sc = workloads.cluttered_room_scene(count, seed, literal=literal)
        tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
        env = None
        if env_size:
            env = crgpu.env_desc(image=workloads.sky_image(width=env_size[0], height=env_size[1], seed=seed + 5))
        out.append((crgpu.GpuScene(tris, sc["materials"], env=env), sc["camera"]))
    return out


def run_batch(args):
    """64 scenes of 10^3-2x10^6 triangles, each job at its own resolution and sample count,
    rendered in one shared pool (autotuned) against one cr_gpu_render after another."""
    import crgpu
    import workloads
    mix = [(c, s, (max(1, int(w * args.mix_scale)), max(1, int(h * args.mix_scale))), spp)
           for c, s, (w, h), spp in workloads.uneven_scene_mix()]
    t0 = time.perf_counter()
    scenes = mix_scenes(literal=args.literal_clutter)
    prep = time.perf_counter() - t0

    def jobs():
        return [crgpu.JobSpec(scenes[i][0], scenes[i][1],
                              crgpu.Options.make(width=w, height=h, samples=spp, bounces=12, seed=42), want_film=False)
                for i, (_, _, (w, h), spp) in enumerate(mix)]

    samples = sum(w * h * spp for _, _, (w, h), spp in mix)
    t0 = time.perf_counter()
    trials = []
    tuning = crgpu.autotune_batch(jobs(), base=crgpu.EngineTuning.make(solo_samples_log2=args.solo_log2), trials=trials)
    tune_s = time.perf_counter() - t0

    def one_by_one_pass():
        # each job through cr_gpu_render_resident, in the same order
        t0 = time.perf_counter()
        for i, (_, _, (w, h), spp) in enumerate(mix):
            scenes[i][0].render_resident(scenes[i][1], crgpu.Options.make(width=w, height=h, samples=spp, bounces=12, seed=42))
        return time.perf_counter() - t0

    for _ in range(max(0, args.warmup)):
        crgpu.render_batch(jobs(), tuning)
        one_by_one_pass()
    # the two arms alternate, step by step, so drifts of the clock or the host hit both alike
    secs, single, est = [], [], None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        est = crgpu.render_batch(jobs(), tuning)
        secs.append(time.perf_counter() - t0)
        single.append(one_by_one_pass())
    value = samples * len(secs) / sum(secs) / 1e6
    single_s = sum(single) / len(single)
    one_by_one = samples / single_s / 1e6
    line = {
        "metric": "aggregate Msamples/s", "value": value, "unit": "Msamples/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded procedural scenes)",
        "config": {"workload": "batch-64-uneven-scenes", "scenes": len(mix), "triangles": int(sum(m[0] for m in mix)),
                   "samples": int(samples), "bounces": 12, "timing": "wall clock around cr_gpu_render_batch",
                   "clutter": "literal config-1 sizes" if args.literal_clutter else "area-preserving sizes",
                   "mix_scale": args.mix_scale},
        "one_by_one": {"value": one_by_one, "unit": "Msamples/s", "seconds": single_s,
                       "step_seconds": [round(x, 3) for x in single]},
        "batch_step_seconds": [round(x, 3) for x in secs],
        "speedup_vs_one_by_one": value / one_by_one,
        "tuning": tuning.as_dict(), "autotune_seconds": tune_s, "autotune_trials": trials, "scene_prep_seconds": prep,
        "engine": est,
    }
    print(json.dumps(line))
    for g, _ in scenes:
        g.close()


def run_serve(args):
    """A Poisson request stream over the 64-scene mix (1024x512 sky per scene) through the
    server: time to the first 4-spp frame and to completion, throughput against the same
    requests rendered as one batch."""
    import crgpu
    import workloads
    stream = [(t, si, (max(1, int(w * args.mix_scale)), max(1, int(h * args.mix_scale))), spp)
              for t, si, (w, h), spp in workloads.request_stream(count=args.requests, rate=args.rate)]
    scenes = mix_scenes(env_size=(1024, 512), literal=args.literal_clutter)

    def spec(r):
        _, si, (w, h), spp = r
        return crgpu.JobSpec(scenes[si][0], scenes[si][1], crgpu.Options.make(width=w, height=h, samples=spp, bounces=12,
                                                                                 seed=42), every=4, fmt=crgpu.ENCODE_SRGB8,
                             want_film=False, keep_frames=False)

    samples = sum(w * h * spp for _, _, (w, h), spp in stream)
    # warm-up: a few requests through a server, then the measured stream
    tuning = crgpu.EngineTuning.make(iterations_per_step=args.engine_iters) if args.engine_iters else None
    srv = crgpu.Server(0, tuning)
    warm = [spec(r) for r in stream[: max(1, args.warmup)]]
    for t in [srv.submit(j) for j in warm]:
        srv.wait(t)
    specs = [spec(r) for r in stream]
    tickets = []
    base = time.perf_counter()
    for r, sp in zip(stream, specs):
        delay = base + r[0] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        tickets.append(srv.submit(sp))
    for t in tickets:
        srv.wait(t)
    sstats = srv.stats()
    srv.close()
    busy = sstats["seconds"]  # the engine's working time (steps), idle waits for arrivals excluded
    sub = np.array([sp.times["submitted"] for sp in specs])
    first = np.array([sp.times["first_frame"] for sp in specs])
    fin = np.array([sp.times["finished"] for sp in specs])
    ok = np.array([sp.status == 0 for sp in specs])
    ttff, ttc = (first - sub)[ok], (fin - sub)[ok]
    served = samples / (fin.max() - sub.min()) / 1e6
    # the same requests as one batch
    t0 = time.perf_counter()
    crgpu.render_batch([spec(r) for r in stream], tuning)
    batched = samples / (time.perf_counter() - t0) / 1e6
    pct = lambda a, q: float(np.percentile(a, q)) * 1e3
    line = {
        "metric": "request latency p50/p99 ms", "value": pct(ttc, 99), "unit": "ms (p99 time-to-completion)",
        "n_gpus": 1, "steps": 1, "warmup": len(warm), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic (seeded procedural scenes, Poisson arrivals)",
        "config": {"workload": "serve-poisson", "requests": len(stream), "rate_per_s": args.rate, "scenes": len(scenes),
                   "env": "1024x512 per scene", "frames": "sRGB8 every 4 spp", "samples": int(samples),
                   "clutter": "literal config-1 sizes" if args.literal_clutter else "area-preserving sizes",
                   "mix_scale": args.mix_scale, "iterations_per_step": args.engine_iters or 8},
        "time_to_first_4spp_ms": {"p50": pct(ttff, 50), "p99": pct(ttff, 99)},
        "time_to_completion_ms": {"p50": pct(ttc, 50), "p99": pct(ttc, 99)},
        "throughput": {"served": served, "batched": batched, "unit": "Msamples/s", "served_over_batched": served / batched,
                       "served_busy": samples / busy / 1e6, "served_busy_over_batched": samples / busy / 1e6 / batched,
                       "note": "served: samples over first arrival to last completion (bounded by the arrival rate "
                               "when the stream offers less than the device renders); served_busy: samples over the "
                               "engine's working time"},
        "offered_load_msamples_per_s": samples / max(1e-9, stream[-1][0]) / 1e6,
        "failed": int((~ok).sum()), "server": sstats,
    }
    print(json.dumps(line))
    for g, _ in scenes:
        g.close()


def _loglog(curve, x):
    """A measured (x, y) curve interpolated in log-log at x; None outside its range."""
    pts = sorted(curve)
    for (x0, y0), (x1, y1) in zip(pts, pts[1:]):
        if x0 <= x <= x1:
            if x1 == x0:
                return y0
            a = (math.log(x) - math.log(x0)) / (math.log(x1) - math.log(x0))
            return math.exp(math.log(y0) + a * (math.log(y1) - math.log(y0)))
    return None


def _time_to(curve, target):
    """Seconds to reach relMSE `target` on a measured (seconds, relMSE) curve, interpolated in
    log-log; None when the curve does not reach it (no extrapolation)."""
    pts = sorted(curve)
    for (t0, e0), (t1, e1) in zip(pts, pts[1:]):
        if e0 >= target >= e1:
            return _loglog([(e1, t1), (e0, t0)], target)
    return None


def run_guided(args):
    """Learned proposal against the plain tracer: relative MSE (against a plain high-sample
    reference) versus wall time, on the caustic sphere grid lit only by the sun disk and on the
    room with next-event estimation off."""
    import crgpu
    import workloads

    def curve(g, cam, make_opt, spps, guided):
        out = []
        for spp in spps:
            gd = crgpu.Guide(seed=1) if guided else None
            t0 = time.perf_counter()
            if guided:
                film, _ = g.render_guided(cam, make_opt(spp), gd, train_samples=min(32, spp))
            else:
                film, _ = g.render(cam, make_opt(spp))
            sec = time.perf_counter() - t0
            out.append((sec, spp, film))
            if gd:
                gd.close()
        return out

    results = {}
    fw, fh = (int(x) for x in args.frame.split("x"))
    for name, sc, (w, h), bounces, nee, spps, ref_spp in (
            ("caustic_sphere_grid", workloads.caustic_scene(fw, fh), (fw, fh), 16, True, (64, 256, 1024, 4096), 16384),
            ("room_without_nee", workloads.room_scene(), (64, 64), 8, False, (256, 1024, 4096), 65536)):
        tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
        env = crgpu.env_desc(image=sc["env_image"]) if sc.get("env_image") is not None else None
        g = crgpu.GpuScene(tris, sc["materials"], env=env)
        cam = sc["camera"]
        make_opt = lambda spp, seed=42: crgpu.Options.make(width=w, height=h, samples=spp, bounces=bounces, seed=seed, nee=nee)
        g.render(cam, make_opt(4))  # warm-up
        t0 = time.perf_counter()
        ref, _ = g.render(cam, make_opt(ref_spp, seed=7))
        ref_s = time.perf_counter() - t0
        entry = {"width": w, "height": h, "bounces": bounces, "nee": nee, "reference_spp": ref_spp,
                 "reference_seconds": ref_s}
        curves = {}
        for label, guided in (("plain", False), ("guided", True)):
            c = curve(g, cam, make_opt, spps, guided)
            pts = [(sec, crgpu.rel_mse(film, ref)) for sec, _, film in c]
            curves[label] = pts
            entry[label] = {"spp": list(spps), "seconds": [p[0] for p in pts], "rel_mse": [p[1] for p in pts],
                            "mean": [float(f.mean()) for _, _, f in c],
                            "seconds_to_rel_mse_1e-3": _time_to(pts, 1e-3)}
        pt, gt = entry["plain"]["seconds_to_rel_mse_1e-3"], entry["guided"]["seconds_to_rel_mse_1e-3"]
        entry["guided_over_plain_time_to_1e-3"] = gt / pt if pt and gt else None
        entry["rel_mse_ratio_at_equal_spp"] = [gq / pq for gq, pq in zip(entry["guided"]["rel_mse"], entry["plain"]["rel_mse"])]
        # guided error over the plain tracer's error after the same wall time (where measured)
        equal_time = []
        for t, e in curves["guided"]:
            p = _loglog(curves["plain"], t)
            equal_time.append(e / p if p else None)
        entry["rel_mse_ratio_at_equal_time"] = equal_time
        results[name] = entry
        g.close()
    c5 = results["caustic_sphere_grid"]
    line = {
        "metric": "time to relMSE 1e-3, guided / plain", "value": c5["guided_over_plain_time_to_1e-3"], "unit": "ratio",
        "note": "null when either tracer does not reach relMSE 1e-3 within the measured samples (no extrapolation)",
        "n_gpus": 1, "steps": 1, "warmup": 1, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64 tracer, fp16 network (fp32 accumulation)", "data": "synthetic (seeded procedural scenes)",
        "config": {"workload": "learned-proposal", "network": "4x64 MLP, 8 vMF lobes, Adam lr 1e-3, trained on the first 32 spp",
                   "guide_probability": 0.5, "reference": "plain tracer, same scene, 16384 spp (room: 65536)"},
        "scenes": results,
    }
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "guided":
        run_guided(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
