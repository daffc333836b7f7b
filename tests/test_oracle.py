"""The CPU restatement (oracle/cr_oracle.cpp) is pinned to the reference: bit-identical
films, per-sample radiance and hits against the reference compiled from its own sources,
and against the committed golden fixtures that the reference produced."""
import numpy as np
import pytest

import scenes
import workloads
from conftest import golden


@pytest.fixture(scope="module")
def oracle():
    import oracle as m
    if not m.available():
        pytest.fail("oracle/liboracle.so is not built (make -f oracle/Makefile)")
    return m


def prepared(crgpu, sc):
    tris, _ = crgpu.finalize(sc["triangles"], sc["materials"], images=sc.get("images", ()), textures=sc.get("textures"))
    return tris, crgpu.build_bvh(tris)


def test_room_film_matches_golden(crgpu, oracle):
    sc = workloads.room_scene()
    tris, bvh = prepared(crgpu, sc)
    film, _, _ = oracle.render_arrays(tris, sc["materials"], bvh, sc["camera"], sc["options"])
    gold = golden("room_film_16spp.npz")
    assert film.tobytes() == gold["film16"].tobytes()


def test_grid_film_matches_golden(crgpu, oracle):
    sc = workloads.sphere_grid_scene(width=192, height=108, samples=4)
    tris, bvh = prepared(crgpu, sc)
    film, _, _ = oracle.render_arrays(tris, sc["materials"], bvh, sc["camera"], sc["options"],
                                      env=crgpu.env_desc(image=sc["env_image"]))
    assert film.tobytes() == golden("grid_film_small.npz")["film"].tobytes()


def test_hits_match_golden(crgpu, oracle):
    import make_golden
    sc = workloads.room_scene()
    tris, bvh = prepared(crgpu, sc)
    gold = golden("hits_room.npz")
    rays = make_golden.room_rays()
    for use_bvh in (True, False):
        f, h = oracle.intersect(tris, sc["materials"], rays, bvh=bvh if use_bvh else None)
        assert np.array_equal(f, gold["found"])
        for k in ("triangle", "t", "u", "v"):
            assert np.array_equal(h[k][f], gold[k][f])
        a, _ = oracle.intersect(tris, sc["materials"], rays, any_hit=True, bvh=bvh if use_bvh else None)
        assert np.array_equal(a, gold["any_found"])


def test_mixed_family_against_reference(crgpu, oracle, ref):
    t, m, images, tex = scenes.bvh_random_scene()
    tris, bvh = prepared(crgpu, dict(triangles=t, materials=m, images=images, textures=tex))
    rays, upper = scenes.bvh_random_rays(tris)
    from crgpu import hit_dtype
    hits = np.zeros(len(rays), hit_dtype)
    hits["t"] = upper
    rs = ref.RefScene(t, m, images=images, textures=tex).build_bvh()
    fr, hr = rs.intersect(rays, hits=hits)
    for use_bvh in (True, False):
        f, h = oracle.intersect(tris, m, rays, hits=hits, bvh=bvh if use_bvh else None, images=images, textures=tex)
        assert np.array_equal(f, fr)
        assert h[f].tobytes() == hr[f].tobytes()


def test_per_sample_streams_and_features_against_reference(crgpu, oracle, ref):
    """Feature fixtures with textures, punctual lights and volumes: films identical to the
    reference's, and every sample's radiance sums to the film."""
    from test_gpu_render import _touching_scene
    sc = _touching_scene()
    tris, bvh = prepared(crgpu, sc)
    import math
    pos = np.array((22, 1, 0), np.float32)
    fwd = scenes.normalize(np.array((20, 2e-6, 0), np.float32) - pos)
    right = scenes.normalize(np.cross(fwd, np.array((0, 1, 0), np.float32)))
    up = np.cross(right, fwd).astype(np.float32)
    cam = crgpu.Camera.make(position=pos, forward=fwd, right=right, up=up, yfov=1e-7)
    o = crgpu.Options.make(width=2, height=2, samples=256, bounces=8, threads=2)
    env = crgpu.env_desc(constant=(1, 1, 1))
    film, per, retries = oracle.render_arrays(tris, sc["materials"], bvh, cam, o, env=env, per_sample=True)
    rf, rst = ref.RefScene(sc["triangles"], sc["materials"]).build_bvh().render(cam, o, ref.RefEnvironment(constant=(1, 1, 1)))
    assert film.tobytes() == rf.tobytes()
    assert retries == rst["boundary_retries"] > 0
    acc = per.astype(np.float64).sum(axis=0)
    assert np.array_equal((acc / o.samples).astype(np.float32), film)


def test_error_text_matches_reference(crgpu, oracle, ref):
    from test_gpu_render import _touching_scene
    sc = _touching_scene()
    tris, bvh = prepared(crgpu, sc)
    bad = crgpu.Camera.make(position=(20, -0.5, 0), forward=(0, 1, 0), right=(1, 0, 0), up=(0, 0, 1), yfov=1e-7)
    o = crgpu.Options.make(width=2, height=2, samples=4, bounces=8, threads=1)
    with pytest.raises(oracle.OracleError) as ours:
        oracle.render_arrays(tris, sc["materials"], bvh, bad, o, env=crgpu.env_desc(constant=(1, 1, 1)), threads=1)
    with pytest.raises(ref.RefError) as theirs:
        ref.RefScene(sc["triangles"], sc["materials"]).build_bvh().render(bad, o, ref.RefEnvironment(constant=(1, 1, 1)))
    assert str(ours.value) == str(theirs.value)
