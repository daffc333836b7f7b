"""Render one of the synthetic workloads on the GPU and print the render statistics as JSON.

The command line the ncu summaries under profiles/ are taken with (one render, no timing
loop around it); bench.py is the measurement.

    python cpu-renderer_b200/render_workload.py --workload grid [--width 1920 --height 1080]
        [--spp 64] [--bounces 16] [--repeat 1] [--exact] [--time-phases] [--count] [--out film.npy]

Workloads: `room` (88 triangles, 256x256, 16 spp, 8 bounces) and `grid` (1,048,576
triangles, 1920x1080, 64 spp, 16 bounces, HDR sky). Sizes default to the workload's own.
"""
import argparse
import json
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import numpy as np  # noqa: E402

import crgpu  # noqa: E402
import workloads  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["room", "grid"], default="grid")
    ap.add_argument("--width", type=int)
    ap.add_argument("--height", type=int)
    ap.add_argument("--spp", type=int)
    ap.add_argument("--bounces", type=int)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--exact", action="store_true", help="FP64 reference-order traversal for every ray")
    ap.add_argument("--time-phases", action="store_true")
    ap.add_argument("--count", action="store_true", help="count node pairs and triangles per closest-hit ray")
    ap.add_argument("--paths-per-wave", type=int, default=0)
    ap.add_argument("--chunk-log2", type=int, default=0, help="2^n sample ids per chunk (0: automatic)")
    ap.add_argument("--out", help="write the film as .npy")
    a = ap.parse_args()
    t0 = time.time()
    sc = workloads.room_scene() if a.workload == "room" else workloads.sphere_grid_scene()
    opt = sc["options"]
    if a.width: opt.width = a.width
    if a.height: opt.height = a.height
    if a.spp: opt.samples = a.spp
    if a.bounces: opt.bounces = a.bounces
    tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
    env = crgpu.env_desc(image=sc["env_image"]) if sc.get("env_image") is not None else None
    g = crgpu.GpuScene(tris, sc["materials"], env=env)
    setup = time.time() - t0
    tun = crgpu.Tuning()
    tun.exact_traversal = int(a.exact)
    tun.time_phases = int(a.time_phases)
    tun.count_traversal = int(a.count)
    tun.paths_per_wave = a.paths_per_wave
    tun.chunk_log2 = a.chunk_log2
    for i in range(a.repeat):
        film, st = g.render(sc["camera"], opt, tuning=tun)
        st["msamples_per_s"] = st["camera_samples"] / st["device_ms"] / 1e3
        st["setup_s"] = setup
        st["workload"] = f"{a.workload} {opt.width}x{opt.height} {opt.samples}spp d{opt.bounces}"
        print(json.dumps(st), flush=True)
    if a.out:
        np.save(a.out, film)


if __name__ == "__main__":
    main()
