"""Generates the committed golden fixtures from the reference itself.

Run in a container where the reference sources are present (oracle/_ref/libcr_ref.so built
by `make -f oracle/Makefile ref`):

    python tests/golden/make_golden.py [--room-spp 4096]

Fixtures (all produced by the UNMODIFIED reference compiled from its sources):
  room_film_4096spp.npz   the 256x256 room workload rendered at 4096 spp (float32 film)
  room_film_16spp.npz     the same at its configured 16 spp, plus per-pixel sample 0 at 1 spp
  hits_room.npz           closest/any hits of seeded random rays in the room scene
  hits_grid.npz           closest hits of seeded rays in the 1,048,576-triangle scene
  grid_film_small.npz     the sphere-grid scene at 192x108, 4 spp
  grid_film_4096spp.npz   the sphere-grid scene (1,048,576 triangles, 2048x1024 sky with the
                          sun) at 192x108, 4096 spp: the acceptance film of the 1080p workload's
                          scene at reduced resolution

    python tests/golden/make_golden.py --only-grid-4096   (that fixture alone)
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "cpu-renderer_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import refimpl  # noqa: E402
import workloads  # noqa: E402
from cr_types import ray_dtype  # noqa: E402


def random_rays(n, lo, hi, seed, y_scale=1.0, y_offset=0.0):
    rng = np.random.default_rng(seed)
    r = np.zeros(n, ray_dtype)
    o = rng.uniform(lo, hi, size=(n, 3))
    o[:, 1] = o[:, 1] * y_scale + y_offset
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r["origin"] = o
    r["direction"] = d
    r["tmin"] = 0
    r["tmax"] = np.inf
    return r


def room_rays():
    return random_rays(4096, -0.95, 0.95, seed=101, y_offset=1.0)


def grid_rays():
    return random_rays(4096, -11.0, 11.0, seed=102, y_scale=0.05, y_offset=0.5)


def grid_4096(threads):
    g = workloads.sphere_grid_scene(width=192, height=108, samples=4096)
    gs = refimpl.RefScene(g["triangles"], g["materials"]).build_bvh()
    genv = refimpl.RefEnvironment(image=g["env_image"])
    gopt = g["options"]
    gopt.threads = threads
    t0 = time.time()
    film, _ = gs.render(g["camera"], gopt, genv)
    print(f"sphere grid 192x108 x 4096 spp: {time.time() - t0:.1f} s on {threads} threads")
    np.savez_compressed(os.path.join(HERE, "grid_film_4096spp.npz"), film=film)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--room-spp", type=int, default=4096)
    ap.add_argument("--skip-room-4096", action="store_true")
    ap.add_argument("--only-grid-4096", action="store_true")
    a = ap.parse_args()
    threads = os.cpu_count()
    if a.only_grid_4096:
        grid_4096(threads)
        return
    sc = workloads.room_scene()
    rs = refimpl.RefScene(sc["triangles"], sc["materials"]).build_bvh()
    env = refimpl.RefEnvironment()
    cam, opt = sc["camera"], sc["options"]
    opt.threads = threads
    film16, _ = rs.render(cam, opt, env)
    opt.samples = 1
    film1, _ = rs.render(cam, opt, env)
    np.savez_compressed(os.path.join(HERE, "room_film_16spp.npz"), film16=film16, film1=film1)
    rays = room_rays()
    f, h = rs.intersect(rays)
    fa, _ = rs.intersect(rays, any_hit=True)
    np.savez_compressed(os.path.join(HERE, "hits_room.npz"), found=f, triangle=h["triangle"], t=h["t"], u=h["u"],
                        v=h["v"], any_found=fa)
    g = workloads.sphere_grid_scene(width=192, height=108, samples=4)
    gs = refimpl.RefScene(g["triangles"], g["materials"]).build_bvh()
    genv = refimpl.RefEnvironment(image=g["env_image"])
    rays = grid_rays()
    f, h = gs.intersect(rays)
    np.savez_compressed(os.path.join(HERE, "hits_grid.npz"), found=f, triangle=h["triangle"], t=h["t"], u=h["u"], v=h["v"])
    gopt = g["options"]
    gopt.threads = threads
    gfilm, _ = gs.render(g["camera"], gopt, genv)
    np.savez_compressed(os.path.join(HERE, "grid_film_small.npz"), film=gfilm)
    if not a.skip_room_4096:
        opt.samples = a.room_spp
        t0 = time.time()
        film, st = rs.render(cam, opt, env)
        print(f"room {a.room_spp} spp: {time.time() - t0:.1f} s on {threads} threads")
        np.savez_compressed(os.path.join(HERE, f"room_film_{a.room_spp}spp.npz"), film=film)


if __name__ == "__main__":
    main()
