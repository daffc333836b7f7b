"""The multi-job engine (cr_gpu_render_batch, cr_server_*): many renders share one path pool.

A job's samples keep their own counter-based streams and its pixel sums are added in sample
order, so every job's film must be bit-identical to the film cr_gpu_render returns for the
same scene, camera and options alone, whatever shares the pool, however the pool is sized,
refilled or stepped. Progressive frames are the encodings of the films at those sample
counts; failures carry the single render's messages and leave the other jobs untouched.
"""
import time

import numpy as np
import pytest

import oracle
import scenes
import workloads
from crgpu import EngineTuning, JobSpec, Server, autotune_batch, render_batch
from test_gpu_render import _touching_scene, gpu_scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def world(crgpu, gpu):
    room = workloads.room_scene()
    rt, _ = crgpu.finalize(room["triangles"], room["materials"])
    grid = workloads.sphere_grid_scene(width=160, height=90, samples=4)
    gt, _ = crgpu.finalize(grid["triangles"], grid["materials"])
    touch = _touching_scene()
    w = dict(
        room=crgpu.GpuScene(rt, room["materials"]),
        room_cam=room["camera"],
        grid=crgpu.GpuScene(gt, grid["materials"], env=crgpu.env_desc(image=grid["env_image"])),
        grid_cam=grid["camera"],
        touch=gpu_scene(crgpu, touch, env=crgpu.env_desc(constant=(1, 1, 1))),
    )
    yield w
    for k in ("room", "grid", "touch"):
        w[k].close()


def _opts(crgpu, w, h, spp, bounces=12, seed=42):
    return crgpu.Options.make(width=w, height=h, samples=spp, bounces=bounces, seed=seed)


def _mixed_jobs(crgpu, world):
    return [
        JobSpec(world["room"], world["room_cam"], _opts(crgpu, 64, 48, 16)),
        JobSpec(world["grid"], world["grid_cam"], _opts(crgpu, 160, 90, 4, seed=7)),
        JobSpec(world["room"], world["room_cam"], _opts(crgpu, 37, 23, 9, bounces=3, seed=1234567)),
        JobSpec(world["grid"], world["grid_cam"], _opts(crgpu, 96, 54, 1)),
        JobSpec(world["room"], world["room_cam"], _opts(crgpu, 128, 128, 2, bounces=8)),
    ]


def _alone(spec):
    film, st = spec.scene.render(spec.camera, spec.options)
    return film, st


@pytest.mark.parametrize("tuning", [
    None,
    dict(pool_paths=4096, range_samples=3000, refill_interval=1, iterations_per_step=4),
    dict(pool_paths=20000, range_samples=1 << 14, refill_interval=3, iterations_per_step=6, use_graphs=0),
    dict(pool_paths=8192, range_samples=2000, issue_policy=2),
    dict(pool_paths=8192, range_samples=5000, refill_free_percent=90),
])
def test_batch_films_equal_single_renders(crgpu, world, tuning):
    jobs = _mixed_jobs(crgpu, world)
    t = EngineTuning.make(**tuning) if tuning else None
    stats = render_batch(jobs, t)
    assert stats["jobs_done"] == len(jobs) and stats["jobs_failed"] == 0
    for i, j in enumerate(jobs):
        assert j.status == 0, j.error
        film, st = _alone(j)
        assert np.array_equal(j.film, film), f"job {i}: relMSE {crgpu.rel_mse(j.film, film)}"
        assert j.stats["camera_samples"] == st["camera_samples"]
        assert j.stats["boundary_retries"] == st["boundary_retries"]
    if tuning and tuning.get("use_graphs", 1):
        assert stats["graph_steps"] > 0


@pytest.mark.parametrize("range_samples", [1024, 1600, 6000])
def test_batch_range_shapes(crgpu, world, range_samples):
    """A job whose samples per pixel fit a range is issued as blocks of pixels holding all their
    samples; one whose samples per pixel exceed it (1536 spp against 1024) as slices of whole
    samples of every pixel. Either shape, and a last block or slice cut short, sums every pixel
    in sample order: films equal the single renders'."""
    jobs = [JobSpec(world["room"], world["room_cam"], _opts(crgpu, 8, 6, 1536, bounces=4)),
            JobSpec(world["grid"], world["grid_cam"], _opts(crgpu, 33, 17, 48, seed=9)),
            JobSpec(world["room"], world["room_cam"], _opts(crgpu, 7, 5, 1, seed=3))]
    stats = render_batch(jobs, EngineTuning.make(pool_paths=4096, range_samples=range_samples, solo_samples_log2=64))
    assert stats["jobs_done"] == len(jobs) and stats["jobs_failed"] == 0
    for i, j in enumerate(jobs):
        assert j.status == 0, j.error
        film, st = _alone(j)
        assert np.array_equal(j.film, film), f"job {i}"
        assert j.stats["camera_samples"] == st["camera_samples"]


def test_batch_solo_jobs(crgpu, world):
    """Jobs of at least 2^solo_samples_log2 samples between two drains render alone through the
    single-render path (here 2^14: the 64x48x16, 160x90x4 and 128x128x2 jobs, and the
    progressive 64x64 job, whose 4-spp frame interval is 2^14 samples), the rest share the pool; every film,
    status and sample count is the standalone render's, and progressive frames and failures
    of solo jobs are reported as for pooled ones."""
    jobs = _mixed_jobs(crgpu, world)
    frames = JobSpec(world["room"], world["room_cam"], _opts(crgpu, 64, 64, 8), every=4, fmt=1)
    bad_cam = crgpu.Camera.make(position=(20, -0.5, 0), forward=(0, 1, 0), right=(1, 0, 0), up=(0, 0, 1), yfov=1e-7)
    failing = JobSpec(world["touch"], bad_cam, _opts(crgpu, 128, 128, 8, bounces=8))
    jobs += [frames, failing]
    stats = render_batch(jobs, EngineTuning.make(pool_paths=8192, range_samples=3000, solo_samples_log2=14))
    assert stats["jobs_done"] == len(jobs) - 1 and stats["jobs_failed"] == 1
    assert stats["camera_samples"] == sum(j.stats["camera_samples"] for j in jobs[:-1])
    for i, j in enumerate(jobs[:-1]):
        assert j.status == 0, j.error
        film, st = _alone(j)
        assert np.array_equal(j.film, film), f"job {i}"
        assert j.stats["camera_samples"] == st["camera_samples"]
        assert j.times["finished"] >= j.times["started"] >= j.times["submitted"]
    assert [s for s, _ in frames.frames] == [4, 8]
    for done, data in frames.frames:
        film, _ = frames.scene.render(frames.camera, _opts(crgpu, 64, 64, done))
        assert data == oracle.encode(film, 1, 0.0), done
    assert frames.times["first_frame"] > 0
    with pytest.raises(crgpu.CrError) as e:
        failing.scene.render(failing.camera, failing.options)
    assert failing.status == e.value.status and failing.error == str(e.value)


def _foliage(crgpu):
    """An alpha-cutout textured quad under a directional light (test_integrator.cpp's foliage
    fixture): a scene that needs the full kernels (alpha test, texture lookups, punctual light)."""
    from crgpu import ALPHA_MASK, WRAP_REPEAT, new_materials, texture_dtype
    m = new_materials(2)
    m[0]["metallic"] = 0; m[0]["base_color"][:3] = (0.4, 0.35, 0.25)
    m[1]["metallic"] = 0; m[1]["double_sided"] = 1; m[1]["alpha_mode"] = ALPHA_MASK
    m[1]["base_color"][:3] = (0.12, 0.45, 0.04)
    images = [np.array([[[1, 1, 1, 1], [1, 1, 1, 0]], [[1, 1, 1, 0], [1, 1, 1, 1]]], np.float32)]
    textures = np.zeros(1, texture_dtype)
    textures[0] = (0, WRAP_REPEAT, WRAP_REPEAT, 0)
    m[1]["base_color_texture"]["texture"] = 0
    tris = scenes.cat(scenes.quad((-8, -0.8, 8), (8, -0.8, 8), (8, -0.8, -8), (-8, -0.8, -8), 0),
                      scenes.quad((-0.8, -0.7, 0), (0.8, -0.7, 0), (0.8, 0.9, 0), (-0.8, 0.9, 0), 1))
    sc = dict(triangles=tris, materials=m, images=images, textures=textures,
              lights=scenes.directional(scenes.normalize((-1, -2, -1)), 2))
    return gpu_scene(crgpu, sc, env=crgpu.env_desc(constant=(0.3, 0.3, 0.3)))


def test_batch_mixing_full_and_lean_scenes(crgpu, world):
    """While a job whose scene has textures, alpha masks and a punctual light is in the pool,
    the steps run the full kernels; once it has ended, the lean ones. Every film is its
    standalone render's either way."""
    foliage = _foliage(crgpu)
    try:
        jobs = [JobSpec(foliage, scenes.room_camera(), _opts(crgpu, 32, 32, 8, bounces=8)),
                JobSpec(world["room"], world["room_cam"], _opts(crgpu, 64, 48, 16)),
                JobSpec(world["grid"], world["grid_cam"], _opts(crgpu, 96, 54, 8, seed=5))]
        stats = render_batch(jobs, EngineTuning.make(pool_paths=4096, range_samples=2048, solo_samples_log2=64))
        assert stats["jobs_done"] == 3
        for i, j in enumerate(jobs):
            assert j.status == 0, j.error
            film, _ = _alone(j)
            assert np.array_equal(j.film, film), f"job {i}"
    finally:
        foliage.close()


def test_batch_progressive_frames(crgpu, world):
    jobs = [JobSpec(world["room"], world["room_cam"], _opts(crgpu, 40, 30, 10), every=4, fmt=0, exposure=0.5),
            JobSpec(world["grid"], world["grid_cam"], _opts(crgpu, 64, 36, 6, seed=3), every=2, fmt=2),
            JobSpec(world["room"], world["room_cam"], _opts(crgpu, 50, 50, 3))]
    render_batch(jobs, EngineTuning.make(pool_paths=4096, range_samples=2500))
    for j, expect, fmt, exposure in ((jobs[0], [4, 8, 10], 0, 0.5), (jobs[1], [2, 4, 6], 2, 0.0)):
        assert j.status == 0, j.error
        assert [s for s, _ in j.frames] == expect
        for done, data in j.frames:
            o = _opts(crgpu, j.options.width, j.options.height, done, seed=j.options.seed)
            film, _ = j.scene.render(j.camera, o)
            assert data == oracle.encode(film, fmt, exposure), done
        assert j.times["first_frame"] > 0
    assert jobs[2].status == 0 and not jobs[2].frames


def test_batch_failures_stay_with_their_jobs(crgpu, world):
    good = JobSpec(world["room"], world["room_cam"], _opts(crgpu, 32, 32, 4))
    o = _opts(crgpu, 2, 2, 64, bounces=8)
    bad_cam = crgpu.Camera.make(position=(20, -0.5, 0), forward=(0, 1, 0), right=(1, 0, 0), up=(0, 0, 1), yfov=1e-7)
    failing = JobSpec(world["touch"], bad_cam, o)
    invalid = JobSpec(world["room"], crgpu.Camera.make(yfov=0.0), _opts(crgpu, 8, 8, 1))
    bad_opts = JobSpec(world["room"], world["room_cam"], crgpu.Options.make(width=0, height=4, samples=1))
    jobs = [good, failing, invalid, bad_opts]
    stats = render_batch(jobs)
    assert stats["jobs_done"] == 1 and stats["jobs_failed"] == 3, [(j.status, j.error) for j in jobs]
    film, _ = _alone(good)
    assert good.status == 0 and np.array_equal(good.film, film)
    for j in (failing, invalid, bad_opts):
        with pytest.raises(crgpu.CrError) as e:
            j.scene.render(j.camera, j.options)
        assert j.status == e.value.status and j.error == str(e.value), (j.error, str(e.value))


def test_server_continuous_batching(crgpu, world):
    """Jobs submitted while others run join the pool; each result is the same as alone."""
    srv = Server(0, EngineTuning.make(pool_paths=1 << 16, range_samples=1 << 14))
    try:
        # a long job first; the others arrive while it is on the GPU and finish before it
        long = JobSpec(world["grid"], world["grid_cam"], _opts(crgpu, 480, 270, 64, seed=11))
        small = _mixed_jobs(crgpu, world) + [
            JobSpec(world["room"], world["room_cam"], _opts(crgpu, 48, 48, 8, seed=99), every=4, fmt=0)]
        jobs = [long] + small
        tickets = [srv.submit(long)]
        time.sleep(0.002)
        tickets += [srv.submit(j) for j in small]
        for t in tickets:
            assert srv.wait(t, 120.0) == 0
        for i, j in enumerate(jobs):
            film, _ = _alone(j)
            assert np.array_equal(j.film, film), f"job {i}"
            tm = j.times
            assert 0 < tm["submitted"] <= tm["started"] <= tm["finished"]
        assert [s for s, _ in jobs[-1].frames] == [4, 8]
        st = srv.stats()
        assert st["jobs_done"] == len(jobs) and st["peak_jobs"] >= 2
        assert min(j.times["finished"] for j in small) < long.times["finished"]
        assert max(j.times["started"] for j in small) < long.times["finished"]
        # a second wave after the engine went idle starts the issue list over
        again = JobSpec(world["grid"], world["grid_cam"], _opts(crgpu, 80, 45, 2, seed=5))
        assert srv.wait(srv.submit(again), 120.0) == 0
        assert np.array_equal(again.film, _alone(again)[0])
    finally:
        srv.close()


def test_server_wait_timeout_and_budget(crgpu, world):
    # a budget that holds one 64x64 job's buffers at a time: jobs run one after another
    per_job = 64 * 64 * 36
    srv = Server(0, EngineTuning.make(pool_paths=1 << 14, memory_budget=per_job + 100))
    try:
        jobs = [JobSpec(world["room"], world["room_cam"], _opts(crgpu, 64, 64, 4, seed=s)) for s in range(3)]
        tickets = [srv.submit(j) for j in jobs]
        for t in tickets:
            assert srv.wait(t, 120.0) == 0
        assert srv.stats()["peak_jobs"] == 1
        for j in jobs:
            assert np.array_equal(j.film, _alone(j)[0])
        big = JobSpec(world["room"], world["room_cam"], _opts(crgpu, 128, 128, 1))
        assert srv.wait(srv.submit(big), 60.0) == 6  # needs more than the budget
        assert "memory budget" in big.error
    finally:
        srv.close()


def test_autotune_picks_a_measured_setting(crgpu, world):
    """The autotuner searches queue depth, regroup interval, refill threshold and block size
    one after another and returns the fastest trial it ran."""
    jobs = _mixed_jobs(crgpu, world)
    trials = []
    t = autotune_batch(jobs, trials=trials)
    assert t.pool_paths in (1 << 22, 1 << 23, 1 << 24, 1 << 25) and t.refill_free_percent in (0, 50, 90)
    assert t.iterations_per_step in (8, 16, 32) and t.block_size in (64, 128, 256)
    assert len(trials) >= 11
    assert {tr["block_size"] for tr in trials} == {64, 128, 256}
    timed = trials[1:]  # the first trial warms the scenes and device blocks
    best = min(timed, key=lambda tr: tr["seconds"])
    assert (t.pool_paths, t.iterations_per_step, t.refill_free_percent, t.block_size) == (
        best["pool_paths"], best["iterations_per_step"], best["refill_free_percent"], best["block_size"])
    stats = render_batch(jobs, t)
    assert stats["jobs_done"] == len(jobs)
    for j in jobs:
        assert np.array_equal(j.film, _alone(j)[0])
