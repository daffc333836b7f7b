"""Output encoding on the device (cr_gpu_encode, cr_gpu_film_encode, cr_gpu_render_progressive)
against the oracle, which tests/test_encode.py pins to the reference's io::writePng pixels and
io::writeHdr files: every byte must match, and failures carry the reference's messages.
"""
import ctypes

import numpy as np
import pytest

import oracle
import workloads
from test_encode import _bad_films, encode_films

pytestmark = pytest.mark.gpu
FORMATS = [0, 1, 2]  # SRGB8, RGBE, HDR file


@pytest.mark.parametrize("name", list(encode_films().keys()))
@pytest.mark.parametrize("fmt", FORMATS)
def test_device_encode_equals_oracle(crgpu, gpu, name, fmt):
    film = encode_films()[name]
    if fmt == 0 and film.max() >= 1e38:
        film = np.minimum(film, np.float32(1e30))
    for exposure in ([0.0, -3.0, 2.5] if fmt == 0 else [0.0]):
        assert crgpu.encode(film, fmt, exposure) == oracle.encode(film, fmt, exposure), (name, exposure)


def test_device_encode_full_hd_film(crgpu, gpu):
    rng = np.random.default_rng(1080)
    film = rng.lognormal(-1, 2, size=(1080, 1920, 3)).astype(np.float32)
    film[500:520] = 0.0
    film[:, 100:300] = film[:, 100:101]
    for fmt in FORMATS:
        assert crgpu.encode(film, fmt, 1.0) == oracle.encode(film, fmt, 1.0), fmt


@pytest.mark.parametrize("case", list(_bad_films().keys()))
@pytest.mark.parametrize("fmt", [0, 2])
def test_device_encode_validation_messages(crgpu, gpu, case, fmt):
    film = _bad_films()[case]
    try:
        oracle.encode(film, fmt)
        expected = None
    except oracle.OracleError as e:
        expected = str(e)
    if expected is None:
        assert crgpu.encode(film, fmt) == oracle.encode(film, fmt)
    else:
        with pytest.raises(crgpu.CrError) as e:
            crgpu.encode(film, fmt)
        assert e.value.status == 1 and str(e.value) == expected


def test_device_encode_capacity_and_dimensions(crgpu, gpu):
    film = np.full((4, 9, 3), 0.5, np.float32)
    size = ctypes.c_uint64(0)
    small = np.zeros(8, np.uint8)
    st = crgpu.lib.cr_gpu_encode(film.ctypes.data, 9, 4, 2, 0.0, 0, small.ctypes.data, 8, ctypes.byref(size))
    assert st == 3 and size.value == len(oracle.encode(film, 2))
    st = crgpu.lib.cr_gpu_encode(film.ctypes.data, 0, 4, 0, 0.0, 0, None, 0, ctypes.byref(size))
    assert st == 1 and "image dimensions must be positive" in crgpu.last_error()


def _room(crgpu, w=48, h=40, spp=12):
    sc = workloads.room_scene()
    tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
    g = crgpu.GpuScene(tris, sc["materials"])
    opt = crgpu.Options.make(width=w, height=h, samples=spp, bounces=8, seed=42)
    return g, sc["camera"], opt


def test_film_encode_after_render(crgpu, gpu):
    g, cam, opt = _room(crgpu)
    film, _ = g.render(cam, opt)
    for fmt in FORMATS:
        assert g.film_encode(fmt, 0.5) == oracle.encode(film, fmt, 0.5)
    g.close()


@pytest.mark.parametrize("fmt", [0, 2])
def test_progressive_frames_are_the_renders_at_those_sample_counts(crgpu, gpu, fmt):
    g, cam, opt = _room(crgpu, spp=10)
    frames, film, stats = g.render_progressive(cam, opt, 4, fmt, 0.0)
    assert [s for s, _ in frames] == [4, 8, 10]
    for done, data in frames:
        o = crgpu.Options.make(width=opt.width, height=opt.height, samples=done, bounces=8, seed=42)
        f, _ = g.render(cam, o)
        assert data == oracle.encode(f, fmt, 0.0), done
    final, _ = g.render(cam, opt)
    assert np.array_equal(film, final)
    assert stats["camera_samples"] == opt.width * opt.height * opt.samples
    g.close()


def test_progressive_rejects_oversized_frames(crgpu, gpu):
    g, cam, _ = _room(crgpu)
    opt = crgpu.Options.make(width=4096, height=4096, samples=32, bounces=2)
    with pytest.raises(crgpu.CrError) as e:
        g.render_progressive(cam, opt, 17)
    assert "every_samples*width*height" in str(e.value)
    g.close()
