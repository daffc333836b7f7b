"""Render parity of the CUDA wavefront tracer against the reference's cr::render
(render.cpp:352-456), with the same counter-based sample streams.

Tolerances. Geometry (camera rays, hits, surface reconstruction) is bit-exact; float and
double arithmetic follows the reference's operation order without FMA, so most samples are
bit-identical. Transcendental functions (cos, sin, pow, exp, log, atan2, acos) are not
bit-reproducible across libm implementations, so a small share of samples diverge by an ulp
and, rarely, take another branch. Films are therefore scored with
relMSE = mean((x - r)^2 / (r^2 + 1e-2)) over pixels and channels: <= 1e-4 at 4096 spp
against the reference CPU render is the acceptance bar; smaller configurations use the
bounds stated in each test."""
import os

import numpy as np
import pytest

import scenes
import workloads
from conftest import golden
from crgpu import INF, Tuning, new_lights, new_materials, LIGHT_DIRECTIONAL, ALPHA_MASK, texture_dtype, WRAP_REPEAT

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 1


def gpu_scene(crgpu, sc, env=None):
    tris, _ = crgpu.finalize(sc["triangles"], sc["materials"], images=sc.get("images", ()), textures=sc.get("textures"))
    return crgpu.GpuScene(tris, sc["materials"], lights=sc.get("lights"), images=sc.get("images", ()),
                          textures=sc.get("textures"), env=env)


def ref_scene(ref, sc):
    return ref.RefScene(sc["triangles"], sc["materials"], lights=sc.get("lights"), images=sc.get("images", ()),
                        textures=sc.get("textures")).build_bvh()


def test_camera_rays_bit_exact(crgpu, ref, gpu):
    sc = workloads.room_scene()
    g = gpu_scene(crgpu, sc)
    cam, opt = sc["camera"], sc["options"]
    W, H = opt.width, opt.height
    for sample in (0, 7):
        rays = g.camera_rays(cam, opt, sample)
        # the reference's jitter: two draws of sampleSeed(seed, pixel, sample) (render.cpp:396-398)
        seeds = np.array([ref.sample_seed(opt.seed, p, sample) for p in range(W * H)], np.uint64)
        def draw(state):
            state = state + np.uint64(0x9E3779B97F4A7C15)
            z = state
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            return state, ((z ^ (z >> np.uint64(31))) >> np.uint64(32)).astype(np.uint32)
        with np.errstate(over="ignore"):
            s, a = draw(seeds)
            s, b = draw(s)
        px = np.float32(np.arange(W * H) % W) + (a >> 8).astype(np.float32) * np.float32(1 / 16777216)
        py = np.float32(np.arange(W * H) // W) + (b >> 8).astype(np.float32) * np.float32(1 / 16777216)
        expected = ref.camera_generate(cam, px.astype(np.float32), py.astype(np.float32), W, H)
        assert rays.tobytes() == expected.tobytes()


def test_room_film_matches_reference(crgpu, ref, gpu):
    sc = workloads.room_scene()
    g = gpu_scene(crgpu, sc)
    cam, opt = sc["camera"], sc["options"]
    opt.threads = THREADS
    film, st = g.render(cam, opt)
    rf, rst = ref_scene(ref, sc).render(cam, opt, ref.RefEnvironment())
    assert st["camera_samples"] == rst["camera_samples"] == 256 * 256 * 16
    assert st["workers"] == rst["workers"]
    assert crgpu.rel_mse(film, rf) < 1e-8
    assert np.mean(np.all(film == rf, axis=2)) > 0.85


def test_room_single_sample_streams(crgpu, gpu):
    """At 1 spp every pixel is exactly one camera sample: most are bit-identical to the
    reference's (committed fixture rendered by the reference)."""
    gold = golden("room_film_16spp.npz")
    assert gold is not None
    sc = workloads.room_scene()
    g = gpu_scene(crgpu, sc)
    cam, opt = sc["camera"], sc["options"]
    film16, _ = g.render(cam, opt)
    assert crgpu.rel_mse(film16, gold["film16"]) < 1e-8
    opt.samples = 1
    film, _ = g.render(cam, opt)
    equal = np.mean(np.all(film == gold["film1"], axis=2))
    assert equal > 0.95, equal


def test_room_4096spp_relmse_against_reference_render(crgpu, gpu):
    """Acceptance: relMSE <= 1e-4 at 4096 spp against the reference CPU render (committed
    fixture rendered by the reference with the same seeds)."""
    gold = golden("room_film_4096spp.npz")
    assert gold is not None
    sc = workloads.room_scene()
    g = gpu_scene(crgpu, sc)
    cam, opt = sc["camera"], sc["options"]
    opt.samples = 4096
    film, st = g.render(cam, opt)
    r = crgpu.rel_mse(film, gold["film"])
    assert r <= 1e-4, r
    assert crgpu.relative_l1(film, gold["film"]) < 5e-4


def test_sphere_grid_small_matches_reference(crgpu, ref, gpu):
    sc = workloads.sphere_grid_scene(width=192, height=108, samples=4)
    g = gpu_scene(crgpu, sc, env=crgpu.env_desc(image=sc["env_image"]))
    film, st = g.render(sc["camera"], sc["options"])
    gold = golden("grid_film_small.npz")
    assert gold is not None
    r = crgpu.rel_mse(film, gold["film"])
    assert r < 1e-4, r


def test_determinism_across_wave_sizes(crgpu, gpu):
    sc = workloads.room_scene()
    g = gpu_scene(crgpu, sc)
    cam, opt = sc["camera"], sc["options"]
    a, _ = g.render(cam, opt)
    b, _ = g.render(cam, opt)
    t = Tuning()
    t.paths_per_wave = 5000  # a small pool: many chunks of 5000 samples
    c, st = g.render(cam, opt, tuning=t)
    assert st["iterations"] > 100 and st["chunks"] > 100
    t.chunk_log2 = 18  # chunks of 2^18 samples through the 5000-slot pool: freed slots are refilled
    d, st = g.render(cam, opt, tuning=t)
    assert st["chunks"] == 4 and st["iterations"] > 100
    assert a.tobytes() == b.tobytes() == c.tobytes() == d.tobytes()


@pytest.mark.parametrize("scene", ["room", "sphere_grid"])
def test_traversals_render_the_same_film(crgpu, gpu, scene):
    """The FP32-box traversal and the FP64 exact traversal find the same hits, so the films
    are identical bit for bit."""
    if scene == "room":
        sc = workloads.room_scene()
        g = gpu_scene(crgpu, sc)
    else:
        sc = workloads.sphere_grid_scene(width=160, height=90, samples=4, bounces=8)
        g = gpu_scene(crgpu, sc, env=crgpu.env_desc(image=sc["env_image"]))
    cam, opt = sc["camera"], sc["options"]
    films = []
    for exact in (0, 1):
        t = Tuning()
        t.exact_traversal = exact
        films.append(g.render(cam, opt, tuning=t)[0].tobytes())
    assert films[0] == films[1]


def test_film_is_the_ordered_double_sum_of_samples(crgpu, gpu):
    sc = workloads.room_scene()
    g = gpu_scene(crgpu, sc)
    cam, opt = sc["camera"], sc["options"]
    opt.width = opt.height = 64
    opt.samples = 5
    _, per = g.render_resident(cam, opt, per_sample=True)
    film = g.film(opt.width, opt.height)
    acc = np.zeros(per.shape[1:], np.float64)
    for s in range(opt.samples):
        acc += per[s].astype(np.float64)
    assert np.array_equal((acc / opt.samples).astype(np.float32), film)


def _energy_plane():
    m = new_materials(1)
    m[0]["metallic"] = 0
    m[0]["base_color"][:3] = 0.6
    m[0]["ior"] = 1
    t = scenes.quad((-20, -20, 0), (20, -20, 0), (20, 20, 0), (-20, 20, 0), 0)
    return dict(triangles=t, materials=m)


def test_constant_sky_albedo_and_mis(crgpu, ref, gpu):
    # test_integrator.cpp:246-255
    sc = _energy_plane()
    env = crgpu.env_desc(constant=(1, 1, 1))
    g = gpu_scene(crgpu, sc, env=env)
    o = crgpu.Options.make(width=16, height=16, samples=512, threads=2, bounces=2, rr=False)
    mis, _ = g.render(scenes.room_camera(), o)
    o.next_event_estimation = 0
    plain, _ = g.render(scenes.room_camera(), o)
    lum = lambda f: float(np.mean(f @ np.array([0.2126, 0.7152, 0.0722], np.float32)))
    assert abs(lum(plain) - 0.6) < 1e-4
    assert abs(lum(mis) - lum(plain)) < 0.012
    rf, _ = ref_scene(ref, sc).render(scenes.room_camera(), o, ref.RefEnvironment(constant=(1, 1, 1)))
    assert crgpu.rel_mse(plain, rf) < 1e-8


def test_emitter_mis_and_camera_visible_emission(crgpu, ref, gpu):
    # test_integrator.cpp:256-271
    sc = _energy_plane()
    m = np.concatenate([sc["materials"], new_materials(1)])
    m[1]["base_color"][:3] = 0; m[1]["metallic"] = 0; m[1]["ior"] = 1; m[1]["emission"] = (2, 1.5, 1)
    t = scenes.cat(sc["triangles"], scenes.quad((-2, -2, 2), (-2, 2, 2), (2, 2, 2), (2, -2, 2), 1))
    sc = dict(triangles=t, materials=m)
    g = gpu_scene(crgpu, sc)
    c = crgpu.Camera.make(position=(0, 0, 1), forward=(0, 0, -1), yfov=0.45)
    o = crgpu.Options.make(width=16, height=16, samples=1024, threads=2, bounces=2, rr=False, nee=False)
    plain, _ = g.render(c, o)
    o.next_event_estimation = 1
    lit, _ = g.render(c, o)
    lum = lambda f: float(np.mean(f @ np.array([0.2126, 0.7152, 0.0722], np.float32)))
    assert lum(lit) > 0.3
    assert abs(lum(lit) - lum(plain)) < 0.018
    rf, _ = ref_scene(ref, sc).render(c, o, ref.RefEnvironment())
    assert crgpu.rel_mse(lit, rf) < 1e-8
    c2 = crgpu.Camera.make(position=(0, 0, 1), forward=(0, 0, 1), right=(-1, 0, 0), yfov=0.45)
    o.samples = 4
    visible, _ = g.render(c2, o)
    assert abs(visible[0, 0, 0] - 2) < 1e-5


@pytest.mark.parametrize("kind", range(5))
def test_reference_feature_fixtures(crgpu, ref, gpu, kind):
    """The five compact scenes of test_integrator.cpp:274-314 (diffuse, metal, water,
    alpha-cutout foliage, lit room) against the reference."""
    m = new_materials(2)
    m[0]["metallic"] = 0; m[0]["base_color"][:3] = (0.4, 0.35, 0.25)
    m[1]["metallic"] = 0; m[1]["base_color"][:3] = (0.55, 0.16, 0.08); m[1]["roughness"] = 0.4
    images, textures, lights = (), None, None
    if kind == 1:
        m[1]["metallic"] = 1; m[1]["base_color"][:3] = (0.9, 0.55, 0.16); m[1]["roughness"] = 0.2
    if kind == 2:
        m[1]["transmission"] = 1; m[1]["thickness"] = 1; m[1]["base_color"][:3] = 1
        m[1]["attenuation_color"] = (0.25, 0.85, 0.7); m[1]["attenuation_distance"] = 2; m[1]["ior"] = 1.333; m[1]["roughness"] = 0.14
    if kind == 3:
        m[1]["double_sided"] = 1; m[1]["alpha_mode"] = ALPHA_MASK; m[1]["base_color"][:3] = (0.12, 0.45, 0.04)
        images = [np.array([[[1, 1, 1, 1], [1, 1, 1, 0]], [[1, 1, 1, 0], [1, 1, 1, 1]]], np.float32)]
        textures = np.zeros(1, texture_dtype)
        textures[0] = (0, WRAP_REPEAT, WRAP_REPEAT, 0)
        m[1]["base_color_texture"]["texture"] = 0
    parts = [scenes.quad((-8, -0.8, 8), (8, -0.8, 8), (8, -0.8, -8), (-8, -0.8, -8), 0)]
    if kind == 3:
        parts.append(scenes.quad((-0.8, -0.7, 0), (0.8, -0.7, 0), (0.8, 0.9, 0), (-0.8, 0.9, 0), 1))
    else:
        parts.append(scenes.cube(1))
    if kind == 4:
        parts.append(scenes.quad((-2, -0.8, -2), (2, -0.8, -2), (2, 3, -2), (-2, 3, -2), 0))
        e = new_materials(1)
        e[0]["emission"] = 5; e[0]["metallic"] = 0; e[0]["base_color"][:3] = 0
        m = np.concatenate([m, e])
        parts.append(scenes.quad((-0.8, 2, -0.8), (0.8, 2, -0.8), (0.8, 2, 0.8), (-0.8, 2, 0.8), 2))
    else:
        lights = scenes.directional(scenes.normalize((-1, -2, -1)), 2)
    sc = dict(triangles=scenes.cat(*parts), materials=m, lights=lights, images=images, textures=textures)
    k = 0.01 if kind == 4 else 0.3
    g = gpu_scene(crgpu, sc, env=crgpu.env_desc(constant=(k, k, k)))
    o = crgpu.Options.make(width=32, height=32, samples=32, bounces=8, threads=1)
    film, _ = g.render(scenes.room_camera(), o)
    rf, _ = ref_scene(ref, sc).render(scenes.room_camera(), o, ref.RefEnvironment(constant=(k, k, k)))
    assert np.isfinite(film).all() and (film >= 0).all()
    assert float(np.mean(film @ np.array([0.2126, 0.7152, 0.0722], np.float32))) > 0.01
    assert crgpu.rel_mse(film, rf) < 1e-5, crgpu.rel_mse(film, rf)


def _slab_pixel(crgpu, ref, triangles, materials, lights, env_const, samples, bounces, nee=True, compare=True):
    sc = dict(triangles=triangles, materials=materials, lights=lights)
    g = gpu_scene(crgpu, sc, env=crgpu.env_desc(constant=env_const))
    cam = crgpu.Camera.make(position=(0, 0, 2), yfov=1e-6)
    o = crgpu.Options.make(width=1, height=1, samples=samples, bounces=bounces, threads=1, seed=42, rr=False, nee=nee)
    film, st = g.render(cam, o)
    if compare:
        rf, _ = ref_scene(ref, sc).render(cam, o, ref.RefEnvironment(constant=env_const))
        assert np.allclose(film, rf, rtol=1e-5, atol=1e-6), (film, rf)
    return film[0, 0]


def test_internal_point_light_beer(crgpu, ref, gpu):
    # test_transport_edges.cpp:68-80
    t, m = scenes.slab()
    l = new_lights(1)
    l[0]["position"] = (0, 0, 0.5); l[0]["intensity"] = 0.01
    absorbing = _slab_pixel(crgpu, ref, t, m, l, (0, 0, 0), 64, 1)
    m2 = m.copy(); m2[0]["attenuation_color"] = 1
    clear = _slab_pixel(crgpu, ref, t, m2, l, (0, 0, 0), 64, 1)
    assert clear[0] > 0.1
    assert np.allclose(absorbing, clear * np.array([np.sqrt(0.5), np.sqrt(0.8), 1]), atol=2e-6)


def test_exterior_directional_light(crgpu, ref, gpu):
    # test_transport_edges.cpp:83-98
    t, m = scenes.slab()
    m = np.concatenate([m, m])
    m[0]["roughness"] = 0
    t = t.copy(); t[2]["material"] = t[3]["material"] = 1
    l = scenes.directional((0, 0, 1), 0.01)
    absorbing = _slab_pixel(crgpu, ref, t, m, l, (0, 0, 0), 2048, 2)
    m2 = m.copy(); m2["attenuation_color"] = 1
    clear = _slab_pixel(crgpu, ref, t, m2, l, (0, 0, 0), 2048, 2)
    assert clear[0] > 0.01
    assert np.allclose(absorbing, clear * np.array([0.5, 0.8, 1]), atol=2e-6)


def test_absorbing_slab_nee_and_bsdf_agree(crgpu, ref, gpu):
    # test_transport_edges.cpp:101-111 (131072 samples of one pixel, 12 bounces)
    t, m = scenes.slab()
    plain = _slab_pixel(crgpu, ref, t, m, None, (1, 1, 1), 131072, 12, nee=False, compare=False)
    mis = _slab_pixel(crgpu, ref, t, m, None, (1, 1, 1), 131072, 12, nee=True, compare=False)
    assert plain[0] > 0.25 and plain[0] < plain[1] < plain[2]
    assert np.allclose(mis, plain, atol=0.008)


def test_enclosed_receiver_energy(crgpu, ref, gpu):
    # test_transport_edges.cpp:158-169
    t, m = scenes.slab()
    m[0]["ior"] = 1; m[0]["attenuation_color"] = 1
    r = new_materials(1)
    r[0]["metallic"] = 0; r[0]["ior"] = 1; r[0]["base_color"][:3] = 0.4
    m = np.concatenate([m, r])
    t = scenes.cat(t, scenes.quad((-99, -99, 0.5), (99, -99, 0.5), (99, 99, 0.5), (-99, 99, 0.5), 1))
    nee = _slab_pixel(crgpu, ref, t, m, None, (1, 1, 1), 4096, 6, nee=True, compare=False)
    bsdf = _slab_pixel(crgpu, ref, t, m, None, (1, 1, 1), 4096, 6, nee=False, compare=False)
    assert np.allclose(nee, 0.4, atol=1e-5)
    assert np.allclose(nee, bsdf, atol=1e-5)


def _touching_scene():
    # test_transport_edges.cpp:115-134
    liquid, opaque = new_materials(2)
    liquid["metallic"] = 0; liquid["transmission"] = 1; liquid["ior"] = 1; liquid["thickness"] = 1
    liquid["attenuation_distance"] = 1; liquid["attenuation_color"] = (0.5, 0.8, 1)
    opaque["metallic"] = 0; opaque["ior"] = 1; opaque["base_color"][:3] = 0.6
    m = np.array([liquid, opaque])
    q = lambda *p, mat=0: scenes.quad(*p, mat, uvs=False)
    t = scenes.cat(q((0, 0, 20), (43, 0, 20), (43, 0, -20), (0, 0, -20)), q((0, -2, -20), (43, -2, -20), (43, -2, 20), (0, -2, 20)),
                   q((0, -2, 20), (43, -2, 20), (43, 0, 20), (0, 0, 20)), q((43, -2, -20), (0, -2, -20), (0, 0, -20), (43, 0, -20)),
                   q((0, -2, -20), (0, -2, 20), (0, 0, 20), (0, 0, -20)), q((43, -2, 20), (43, -2, -20), (43, 0, -20), (43, 0, 20)),
                   q((-1, -1, 21), (44, -1, 21), (44, -1, -21), (-1, -1, -21), mat=1))
    touching = crgpu_new_triangle(((19, -1 + 2e-6, -1), (21, 1 + 2e-6, -1), (20, 2e-6, 1)), 1)
    return dict(triangles=scenes.cat(t, touching), materials=m)


def crgpu_new_triangle(points, material):
    from crgpu import new_triangles
    t = new_triangles(1)
    t[0]["v"]["position"] = np.array(points, np.float32)
    t[0]["material"] = material
    return t


def test_precision_replay_and_invalid_camera(crgpu, ref, gpu):
    # test_transport_edges.cpp:115-153
    sc = _touching_scene()
    g = gpu_scene(crgpu, sc, env=crgpu.env_desc(constant=(1, 1, 1)))
    pos = np.array((22, 1, 0), np.float32)
    fwd = scenes.normalize(np.array((20, 2e-6, 0), np.float32) - pos)
    right = scenes.normalize(np.cross(fwd, np.array((0, 1, 0), np.float32)))
    up = np.cross(right, fwd).astype(np.float32)
    cam = crgpu.Camera.make(position=pos, forward=fwd, right=right, up=up, yfov=1e-7)
    o = crgpu.Options.make(width=2, height=2, samples=256, bounces=8, threads=2)
    film, st = g.render(cam, o)
    assert st["boundary_retries"] > 0
    assert np.isfinite(film).all() and (film >= 0).all()
    again, st2 = g.render(cam, o)
    assert st2["boundary_retries"] == st["boundary_retries"] and again.tobytes() == film.tobytes()
    rf, rst = ref_scene(ref, sc).render(cam, o, ref.RefEnvironment(constant=(1, 1, 1)))
    assert crgpu.rel_mse(film, rf) < 1e-3
    bad = crgpu.Camera.make(position=(20, -0.5, 0), forward=(0, 1, 0), right=(1, 0, 0), up=(0, 0, 1), yfov=1e-7)
    with pytest.raises(crgpu.CrError) as e:
        g.render(bad, o)
    assert "outside closed volumes" in str(e.value)
    assert str(e.value).startswith("Pixel (")
    with pytest.raises(ref.RefError) as r:
        ref_scene(ref, sc).render(bad, o, ref.RefEnvironment(constant=(1, 1, 1)))
    assert str(e.value) == str(r.value)


def test_invalid_options_and_camera(crgpu, gpu):
    g = gpu_scene(crgpu, _energy_plane())
    o = crgpu.Options.make(width=0)
    with pytest.raises(crgpu.CrError) as e:
        g.render(scenes.room_camera(), o)
    assert str(e.value) == "Width and height must be in [1, 16384]"
    cam = crgpu.Camera.make(yfov=0.0)
    with pytest.raises(crgpu.CrError) as e:
        g.render(cam, crgpu.Options.make(width=8, height=8, samples=1))
    assert str(e.value) == "Pixel (0,0), sample 0: Invalid perspective camera or image dimensions"


def test_progress_callback(crgpu, gpu):
    g = gpu_scene(crgpu, _energy_plane())
    calls = []
    o = crgpu.Options.make(width=32, height=32, samples=8)
    g.render(scenes.room_camera(), o, progress=lambda a, b, s: calls.append((a, b)))
    assert calls and calls[-1] == (32 * 32 * 8, 32 * 32 * 8)
