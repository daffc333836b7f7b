"""Closest-hit and any-hit parity of the CUDA traversal against the reference's
Bvh::intersect (geometry.cpp:554-639): identical found flags, triangle IDs, and the double
t, u, v of every hit, bit for bit. Families follow tests/test_geometry.cpp:396-658 (brute
force comparisons, ties, adversarial depth, reciprocal slabs, empty BVH, ignoreTriangle,
sub-float ordering, split origins). Every case runs the fast (FP32-box) traversal and the
exact (FP64, reference-order) traversal."""
import numpy as np
import pytest

import scenes
import workloads
from conftest import golden
from crgpu import INF, NO_TRIANGLE, Tuning, hit_dtype, new_materials

pytestmark = pytest.mark.gpu
MODES = [0, 1]


def tuning(exact):
    t = Tuning()
    t.exact_traversal = exact
    return t


def assert_hits_equal(fa, ha, fb, hb, label=""):
    assert np.array_equal(fa, fb), f"{label}: found differs at {np.where(fa != fb)[0][:10]}"
    m = fa
    for k in ("triangle", "t", "u", "v"):
        bad = np.where(m & (ha[k] != hb[k]))[0]
        assert len(bad) == 0, f"{label}: {k} differs at {bad[:10]}: {ha[k][bad[:3]]} vs {hb[k][bad[:3]]}"
    # misses keep the incoming hit untouched, as the reference does
    assert np.array_equal(ha[~m].tobytes() if (~m).any() else b"", hb[~m].tobytes() if (~m).any() else b"")


def both(crgpu, ref, triangles, materials, images=(), textures=None, use_ref_bvh=False):
    tris, _ = crgpu.finalize(triangles, materials, images=images, textures=textures)
    rs = ref.RefScene(triangles, materials, images=images, textures=textures).build_bvh()
    bvh = rs.bvh_arrays() if use_ref_bvh else None
    g = crgpu.GpuScene(tris, materials, images=images, textures=textures, bvh=bvh)
    return g, rs


def compare(g, rs, rays, upper=None, exact=0, label="", ignore=NO_TRIANGLE):
    hits = np.zeros(len(rays), hit_dtype)
    hits["t"] = INF if upper is None else upper
    hits["u"], hits["v"], hits["triangle"] = 0.123, 0.234, 999999
    fa, ha = g.intersect(rays, hits=hits, tuning=tuning(exact), ignore=ignore)
    fb, hb = rs.intersect(rays, hits=hits, ignore=ignore)
    assert_hits_equal(fa, ha, fb, hb, label)
    aa, _ = g.intersect(rays, any_hit=True, hits=hits, tuning=tuning(exact), ignore=ignore)
    ab, _ = rs.intersect(rays, any_hit=True, hits=hits, ignore=ignore)
    assert np.array_equal(aa, ab), f"{label}: any-hit differs at {np.where(aa != ab)[0][:10]}"
    return fa


@pytest.mark.parametrize("exact", MODES)
def test_mixed_material_random_family(crgpu, ref, gpu, exact):
    t, m, images, tex = scenes.bvh_random_scene()
    g, rs = both(crgpu, ref, t, m, images, tex)
    rays, upper = scenes.bvh_random_rays(crgpu.finalize(t, m, images=images, textures=tex)[0])
    found = compare(g, rs, rays, upper, exact, "random family")
    assert found.sum() > 1000


@pytest.mark.parametrize("exact", MODES)
def test_uploading_the_references_own_bvh(crgpu, ref, gpu, exact):
    t, m, images, tex = scenes.bvh_random_scene(seed=3)
    g, rs = both(crgpu, ref, t, m, images, tex, use_ref_bvh=True)
    rays, upper = scenes.bvh_random_rays(crgpu.finalize(t, m, images=images, textures=tex)[0], seed=4, count=3000)
    compare(g, rs, rays, upper, exact, "reference BVH")


@pytest.mark.parametrize("exact", MODES)
def test_index_ties(crgpu, ref, gpu, exact):
    # test_geometry.cpp:572-591: overlapping copies resolve to the lowest index
    m = new_materials(1)
    m[0]["double_sided"] = 1
    g, rs = both(crgpu, ref, scenes.cat(*[scenes.tri() for _ in range(100)]), m)
    found = compare(g, rs, scenes.rays((0.25, 0.25, 1), (0, 0, -1)), exact=exact, label="overlap")
    assert found.all()
    for shift in range(-5, 6):
        x = float(shift)
        target = scenes.tri((x, 0, 0), (x + 1, 0, 0), (x, 1, 0))
        others = [scenes.tri((ox, 0, -2), (ox + 1, 0, -2), (ox, 1, -2)) for ox in (float(((i * 23) % 61 - 30) * 2) for i in range(60))]
        g, rs = both(crgpu, ref, scenes.cat(target, target, *others), m)
        f = compare(g, rs, scenes.rays((x + 0.25, 0.25, 1), (0, 0, -25)), exact=exact, label=f"tie {shift}")
        assert f.all()


@pytest.mark.parametrize("exact", MODES)
def test_exponential_depth(crgpu, ref, gpu, exact):
    m = new_materials(1)
    m[0]["double_sided"] = 1
    ts = [scenes.tri((np.ldexp(1.0, e), 0, 0), (np.ldexp(1.0, e), 1, 0), (np.ldexp(1.0, e), 0, 1)) for e in range(-80, 80)]
    g, rs = both(crgpu, ref, scenes.cat(*ts), m)
    o = [(np.ldexp(1.0, e), 0.25, 0.25) for e in range(-75, 75, 3)]
    compare(g, rs, scenes.rays(o, (-1, 0, 0)), exact=exact, label="exponential")


@pytest.mark.parametrize("exact", MODES)
@pytest.mark.parametrize("scale", [1e-15, 1e-5, 1.0, 1e5, 1e15])
def test_reciprocal_slabs(crgpu, ref, gpu, exact, scale):
    m = new_materials(1)
    m[0]["double_sided"] = 1
    s = np.float32(scale)
    ts = [scenes.tri((np.float32(i) * 5 * s, 0, 0), (np.float32(i) * 5 * s + s, 0, 0), (np.float32(i) * 5 * s, s, 0)) for i in range(20)]
    g, rs = both(crgpu, ref, scenes.cat(*ts), m)
    pts = [(0, 0, s), (s, 0, s), (np.float32(0.5) * s, np.float32(0.5) * s, s)]
    for speed in (1e-30, 1.0, 1e30):
        for negz in (-0.0, 0.0):
            r = scenes.rays(pts, (0, negz, -np.float32(speed)))
            compare(g, rs, r, exact=exact, label=f"slabs {scale} {speed}")
            compare(g, rs, r, upper=0.0, exact=exact, label=f"zero interval {scale} {speed}")


@pytest.mark.parametrize("exact", MODES)
def test_ignore_triangle_and_close_surfaces(crgpu, ref, gpu, exact):
    # test_geometry.cpp:625-637
    m = new_materials(1)
    m[0]["double_sided"] = 1
    t = scenes.cat(scenes.tri((19, 1e-7, -1), (21, 1e-7, -1), (20, 1e-7, 1)), scenes.tri((18, 0, -2), (20, 0, 2), (22, 0, -2)))
    g, rs = both(crgpu, ref, t, m)
    r = scenes.rays((20, 1e-7, 0), (0, -1, 0))
    f = compare(g, rs, r, exact=exact, label="self")
    assert f.all()
    f = compare(g, rs, r, exact=exact, label="ignore 0", ignore=0)
    assert f.all()


@pytest.mark.parametrize("exact", MODES)
def test_sub_float_ordering_and_split_origins(crgpu, ref, gpu, exact):
    m = new_materials(1)
    t = scenes.cat(scenes.tri(), scenes.tri((0, 0, 1e-6), (1, 0, 1e-6), (0, 1, 1e-6)))
    g, rs = both(crgpu, ref, t, m)
    f = compare(g, rs, scenes.rays((0.25, 0.25, 100), (0, 0, -1)), exact=exact, label="sub-float")
    assert f.all()
    g, rs = both(crgpu, ref, scenes.tri(), new_materials(1))
    r = scenes.rays((0.25, 0.25, 1), (0, 0, -1), low=(0, 0, 1e-9))
    compare(g, rs, r, exact=exact, label="split origin")


def test_empty_scene(crgpu, ref, gpu):
    g = crgpu.GpuScene(np.zeros(0, crgpu.triangle_dtype), new_materials(1))
    f, h = g.intersect(scenes.rays((0, 0, 1), (0, 0, -1)))
    assert not f.any() and h["t"][0] == INF


@pytest.mark.parametrize("exact", MODES)
def test_invalid_rays_are_rejected(crgpu, ref, gpu, exact):
    g, rs = both(crgpu, ref, scenes.tri(), new_materials(1))
    nan = np.float32(np.nan)
    r = np.concatenate([scenes.rays((nan, 0, 1), (0, 0, -1)), scenes.rays((0.25, 0.25, 1), (0, nan, -1)),
                        scenes.rays((0.25, 0.25, 1), (0, 0, -1), tmin=nan), scenes.rays((0.25, 0.25, 1), (0, 0, 0)),
                        scenes.rays((0.25, 0.25, 1), (0, 0, -1), tmin=2, tmax=1),
                        scenes.rays((np.inf, 0, 1), (0, 0, -1))])
    f = compare(g, rs, r, exact=exact, label="invalid")
    assert not f.any()


@pytest.mark.parametrize("exact", MODES)
def test_workload_rays(crgpu, ref, gpu, exact):
    import make_golden
    sc = workloads.room_scene()
    g, rs = both(crgpu, ref, sc["triangles"], sc["materials"])
    compare(g, rs, make_golden.room_rays(), exact=exact, label="room rays")
    cr = g.camera_rays(sc["camera"], sc["options"], 3)
    compare(g, rs, cr, exact=exact, label="room camera rays")


@pytest.mark.parametrize("exact", MODES)
def test_million_triangle_scene(crgpu, ref, gpu, exact):
    import make_golden
    sc = workloads.sphere_grid_scene(width=192, height=108, samples=1, sky=False)
    g, rs = both(crgpu, ref, sc["triangles"], sc["materials"])
    rays = make_golden.grid_rays()
    f = compare(g, rs, rays, exact=exact, label="grid rays")
    assert f.sum() > 500
    cr = g.camera_rays(sc["camera"], sc["options"], 0)
    compare(g, rs, cr, exact=exact, label="grid camera rays")


def test_golden_hits_without_reference(crgpu, gpu):
    """The committed fixtures (produced by the reference) also pin the traversal."""
    import make_golden
    for name, sc, rays in (("hits_room.npz", workloads.room_scene(), make_golden.room_rays()),
                           ("hits_grid.npz", workloads.sphere_grid_scene(sky=False), make_golden.grid_rays())):
        gold = golden(name)
        assert gold is not None, name
        tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
        g = crgpu.GpuScene(tris, sc["materials"])
        f, h = g.intersect(rays)
        assert np.array_equal(f, gold["found"])
        for k in ("triangle", "t", "u", "v"):
            assert np.array_equal(h[k][f], gold[k][f]), k
        if "any_found" in gold:
            a, _ = g.intersect(rays, any_hit=True)
            assert np.array_equal(a, gold["any_found"])
