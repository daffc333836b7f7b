"""Scene-upload validation (cr_gpu_scene_create). The upload runs the triangle copy and the
environment tables on helper threads beside the geometry checks; an error raised on any of
them must reach the caller with the reference's message, in the order the checks have in a
sequential upload (geometry before environment), and leave the device usable."""
import numpy as np
import pytest

import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def room(crgpu, gpu):
    sc = workloads.room_scene()
    tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
    nodes, idx = crgpu.build_bvh(tris)
    return sc, tris, nodes, idx


def _sky(bad=False):
    img = np.ones((64, 128, 4), np.float32)
    if bad:
        img[10, 20, 1] = -1.0
    return img


def _create(crgpu, sc, tris, env=None, bvh=None, materials=None):
    return crgpu.GpuScene(tris, sc["materials"] if materials is None else materials, env=env, bvh=bvh)


def test_negative_sky_pixel_is_reported(crgpu, room):
    sc, tris, nodes, idx = room
    with pytest.raises(crgpu.CrError, match="Non-finite or negative HDR environment pixel"):
        _create(crgpu, sc, tris, env=crgpu.env_desc(image=_sky(bad=True)), bvh=(nodes, idx))


def test_material_index_out_of_range_is_reported(crgpu, room):
    sc, tris, nodes, idx = room
    bad = tris.copy()
    bad["material"][3] = len(sc["materials"])
    with pytest.raises(crgpu.CrError, match="Triangle material index out of range"):
        _create(crgpu, sc, bad, env=crgpu.env_desc(image=_sky()))


def test_bvh_error_comes_before_the_environment_error(crgpu, room):
    """A malformed BVH is found while both helpers run; with a bad sky as well, the BVH error
    is the one reported, as in a sequential upload."""
    sc, tris, nodes, idx = room
    broken = nodes.copy()
    interior = np.where(broken["count"] == 0)[0]
    broken["first"][interior[0]] += 1  # an even first child: not an adjacent pair
    message = "BVH interior node does not reference an adjacent child pair"
    with pytest.raises(crgpu.CrError, match=message):
        _create(crgpu, sc, tris, env=crgpu.env_desc(image=_sky()), bvh=(broken, idx))
    with pytest.raises(crgpu.CrError, match=message):
        _create(crgpu, sc, tris, env=crgpu.env_desc(image=_sky(bad=True)), bvh=(broken, idx))


def test_scenes_render_after_failed_uploads(crgpu, room):
    sc, tris, nodes, idx = room
    for _ in range(2):
        with pytest.raises(crgpu.CrError):
            _create(crgpu, sc, tris, env=crgpu.env_desc(image=_sky(bad=True)), bvh=(nodes, idx))
    g = _create(crgpu, sc, tris, env=crgpu.env_desc(image=_sky()), bvh=(nodes, idx))
    o = crgpu.Options.make(width=32, height=32, samples=2, bounces=4)
    film, _ = g.render(sc["camera"], o)
    ref = _create(crgpu, sc, tris, env=crgpu.env_desc(image=_sky()))
    film2, _ = ref.render(sc["camera"], o)
    assert np.isfinite(film).all() and np.array_equal(film, film2)
    g.close()
    ref.close()
