"""Guided renders (cr_gpu_render_guided): the network trained online on the tracer's own samples
and mixed with BSDF sampling by one-sample MIS.

* The estimator stays unbiased: with next-event estimation on (MIS weights with the mixture's
  density), the guided film converges to the plain film.
* The trained network gains: on the room with next-event estimation off, where emitters are
  found only by sampled directions, a guided render has a clearly lower error than a plain
  render with the same samples.
* The estimator stays unbiased under an HDR sky: on the learned-proposal scene (smooth
  dielectric and sharp conductor spheres lit only by a 5e4 sun disk, whose bilinear halo is a
  heavy-tailed light source), the guided film's mean lies within the plain tracer's own
  seed-to-seed spread of the reference's.
"""
import numpy as np
import pytest

import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def room(crgpu, gpu):
    sc = workloads.room_scene()
    tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
    g = crgpu.GpuScene(tris, sc["materials"])
    yield g, sc["camera"]
    g.close()


def _opt(crgpu, spp, seed=42, nee=True):
    return crgpu.Options.make(width=64, height=64, samples=spp, bounces=8, seed=seed, nee=nee)


def test_guided_estimator_is_unbiased(crgpu, room):
    g, cam = room
    ref, _ = g.render(cam, _opt(crgpu, 32768, seed=9))
    plain, _ = g.render(cam, _opt(crgpu, 1024))
    gd = crgpu.Guide(seed=2)
    guided, st = g.render_guided(cam, _opt(crgpu, 1024), gd)
    assert st["camera_samples"] == 64 * 64 * 1024
    assert np.isfinite(guided).all() and (guided >= 0).all()
    assert guided.mean() == pytest.approx(ref.mean(), rel=0.01)
    assert crgpu.rel_mse(guided, ref) < 2.0 * crgpu.rel_mse(plain, ref)
    gd.close()


def test_trained_guide_lowers_the_error_without_nee(crgpu, room):
    g, cam = room
    ref, _ = g.render(cam, _opt(crgpu, 65536, seed=9, nee=False))
    plain, _ = g.render(cam, _opt(crgpu, 256, nee=False))
    gd = crgpu.Guide(seed=1)
    guided, _ = g.render_guided(cam, _opt(crgpu, 256, nee=False), gd, train_samples=32)
    e_plain, e_guided = crgpu.rel_mse(plain, ref), crgpu.rel_mse(guided, ref)
    print(f"relMSE at 256 spp: plain {e_plain:.4f}, guided {e_guided:.4f}")
    assert e_guided < 0.8 * e_plain
    assert guided.mean() == pytest.approx(ref.mean(), rel=0.02)
    gd.close()


def test_guide_keeps_its_training(crgpu, room):
    """The guide passed to a render is trained by it; a second render continues from there."""
    g, cam = room
    gd = crgpu.Guide(seed=3)
    before = gd.parameters()
    g.render_guided(cam, _opt(crgpu, 8, nee=False), gd, train_samples=8)
    after = gd.parameters()
    assert not np.array_equal(before, after)
    g.render_guided(cam, _opt(crgpu, 4, nee=False), gd, train_samples=0)  # no training: weights kept
    assert np.array_equal(after, gd.parameters())
    gd.close()


def test_guided_estimator_is_unbiased_under_the_sun(crgpu, gpu):
    sc = workloads.caustic_scene(width=32, height=18, samples=1)
    tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
    g = crgpu.GpuScene(tris, sc["materials"], env=crgpu.env_desc(image=sc["env_image"]))
    cam = sc["camera"]

    def opt(spp, seed):
        return crgpu.Options.make(width=32, height=18, samples=spp, bounces=16, seed=seed)

    ref = g.render(cam, opt(262144, 99))[0].astype(np.float64).mean()
    plain = [g.render(cam, opt(16384, seed))[0].astype(np.float64).mean() for seed in range(1, 7)]
    sigma = float(np.std(plain, ddof=1))
    gd = crgpu.Guide(seed=6)
    guided_film, _ = g.render_guided(cam, opt(16384, 42), gd)
    guided = guided_film.astype(np.float64).mean()
    print(f"film mean: reference {ref:.5f}, plain {np.mean(plain):.5f} +- {sigma:.5f}, guided {guided:.5f}")
    assert np.isfinite(guided_film).all() and (guided_film >= 0).all()
    assert abs(guided - ref) < 5 * sigma + 0.01 * ref
    gd.close()
    g.close()
