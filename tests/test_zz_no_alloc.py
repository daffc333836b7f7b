"""cr_gpu_render_noalloc: the render entry point that allocates nothing.

Some callers cannot allocate device memory while they render: hosts that hand out GPU
memory only at start-up, request paths that must not block on cudaMalloc/cudaFree (both can
synchronise the device or fail under memory pressure), and code sharing a device it must not
fragment. For them the library keeps one fixed 32 MiB workspace per device. These checks call
the entry point through the C ABI and compare it with cr_gpu_render on the same scene: the
films must be identical (the same kernels, sample streams and ordered FP64 sums), on two
calls in a row, since the workspace keeps the previous call's contents and every call must
clear what has to start at zero.

This file is collected last so that a run stopping at the first failure has already run the
other tests; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest

import workloads

pytestmark = pytest.mark.gpu


def render_noalloc(crgpu, scene, camera, options):
    film = np.zeros((options.height, options.width, 3), np.float32)
    stats = crgpu.Stats()
    status = crgpu.lib.cr_gpu_render_noalloc(scene.handle, ctypes.byref(camera), ctypes.byref(options),
                                             film.ctypes.data, ctypes.byref(stats))
    return status, film, stats.as_dict()


def test_noalloc_render_matches_cr_gpu_render_twice(crgpu, gpu):
    sc = workloads.room_scene()
    tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
    g = crgpu.GpuScene(tris, sc["materials"])
    cam, opt = sc["camera"], sc["options"]
    expected, st = g.render(cam, opt)
    for call in range(2):
        before = crgpu.allocation_count()
        status, film, stats = render_noalloc(crgpu, g, cam, opt)
        assert status == 0, crgpu.last_error()
        # the property the entry point exists for: the library requested no memory block
        assert crgpu.allocation_count() == before, f"call {call} allocated"
        assert stats["camera_samples"] == st["camera_samples"]
        assert stats["device_ms"] > 0
        assert np.array_equal(film, expected), f"call {call}: relMSE {crgpu.rel_mse(film, expected)}"


def test_noalloc_render_with_environment_and_several_chunks(crgpu, gpu):
    # 192x108 x 32 spp = 663,552 samples: more than one 524,288-sample chunk of the workspace
    sc = workloads.sphere_grid_scene(width=192, height=108, samples=32)
    tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
    g = crgpu.GpuScene(tris, sc["materials"], env=crgpu.env_desc(image=sc["env_image"]))
    expected, _ = g.render(sc["camera"], sc["options"])
    for call in range(2):
        before = crgpu.allocation_count()
        status, film, stats = render_noalloc(crgpu, g, sc["camera"], sc["options"])
        assert status == 0, crgpu.last_error()
        assert crgpu.allocation_count() == before, f"call {call} allocated"
        assert stats["chunks"] == 2
        assert np.array_equal(film, expected), f"call {call}"


def test_noalloc_rejects_images_beyond_its_workspace(crgpu, gpu):
    sc = workloads.room_scene()
    tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
    g = crgpu.GpuScene(tris, sc["materials"])
    opt = crgpu.Options.make(width=513, height=512, samples=1, bounces=2)
    status, _, _ = render_noalloc(crgpu, g, sc["camera"], opt)
    assert status == 1
    assert "262144 pixels" in crgpu.last_error()
    # the failed call leaves the workspace usable
    opt = sc["options"]
    expected, _ = g.render(sc["camera"], opt)
    status, film, _ = render_noalloc(crgpu, g, sc["camera"], opt)
    assert status == 0 and np.array_equal(film, expected)
