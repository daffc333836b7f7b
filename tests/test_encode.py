"""Output encoding, CPU side: the oracle's restatement of io::writePng's display mapping and of
io::writeHdr's Radiance writer (stb_image_write 1.16) is pinned against the reference's own
writers (oracle/_ref/libcr_ref.so: src/io/image.cpp with its vendored codec), and the
product's display-threshold table (cr_display_thresholds, used by the device encoder) is
checked against the direct mapping.
"""
import os

import numpy as np
import pytest

import crgpu
import imagefile
import oracle

FLT_MAX = np.float32(3.4028234663852886e38)


def encode_films():
    """Films that exercise every branch of the writers (seeded)."""
    rng = np.random.default_rng(0x5EED0E0C)
    films = {}
    films["lognormal_53x37"] = rng.lognormal(0, 2, size=(37, 53, 3)).astype(np.float32)
    # runs: constant rows longer than 127 and 128, literal stretches longer than 128
    f = rng.lognormal(0, 1, size=(6, 300, 3)).astype(np.float32)
    f[0] = 1.0
    f[1, :200] = 0.25
    f[2, 10:13] = 3.0
    f[3, ::2] = 0.0
    f[4] = 0.0
    films["runs_300x6"] = f
    # widths below 8 take the flat (no run-length) branch
    films["narrow_7x5"] = rng.lognormal(0, 1, size=(5, 7, 3)).astype(np.float32)
    films["single_1x1"] = np.array([[[0.5, 2.0, 0.0]]], np.float32)
    films["width8_8x3"] = rng.lognormal(0, 1, size=(3, 8, 3)).astype(np.float32)
    # extremes: tiny (< 1e-32), subnormal, below 2^127, mantissas at 1 - 2^-24
    e = np.zeros((4, 16, 3), np.float32)
    e[0, :, 0] = np.float32(1e-33)
    e[0, :, 1] = np.float32(1e-40)
    e[1] = np.float32(1.7e38)
    mant = np.float32(1 - 2.0 ** -24)
    e[2] = (mant * np.float32(2.0) ** rng.integers(-60, 60, size=(16, 1))).astype(np.float32)
    e[3, :, 0] = mant * 8
    e[3, :, 1] = 7.9999995
    e[3, :, 2] = 4.0000005
    films["extremes_16x4"] = e
    return films


@pytest.fixture(scope="module")
def films():
    return encode_films()


@pytest.mark.parametrize("name", list(encode_films().keys()))
def test_oracle_hdr_file_is_reference_writehdr(ref, films, name, tmp_path):
    film = films[name]
    path = tmp_path / "ref.hdr"
    ref.write_hdr(path, film)
    assert oracle.encode(film, crgpu.ENCODE_HDR_FILE) == path.read_bytes()


@pytest.mark.parametrize("exposure", [0.0, -3.0, 2.5, 24.0, -24.0])
def test_oracle_display_bytes_are_reference_writepng(ref, films, exposure, tmp_path):
    for name, film in films.items():
        if film.max() >= 1e38:
            continue
        path = tmp_path / f"{name}.png"
        ref.write_png(path, film, exposure)
        png = imagefile.read_png(path)
        got = np.frombuffer(oracle.encode(film, crgpu.ENCODE_SRGB8, exposure), np.uint8).reshape(png.shape)
        assert np.array_equal(got, png), name


def _bad_films():
    good = np.full((2, 3, 3), 0.5, np.float32)
    out = {}
    for label, value in [("nan", np.nan), ("inf", np.inf), ("negative", -1e-6), ("huge", 2.0 ** 127)]:
        f = good.copy()
        f[1, 2, 1] = value
        out[label] = f
    f = good.copy()  # a later invalid pixel after an out-of-range one: the first wins
    f[0, 1, 0] = 2.0 ** 127
    f[1, 0, 2] = np.nan
    out["huge_then_nan"] = f
    return out


@pytest.mark.parametrize("fmt", [crgpu.ENCODE_SRGB8, crgpu.ENCODE_HDR_FILE])
@pytest.mark.parametrize("case", list(_bad_films().keys()))
def test_oracle_validation_messages_are_the_reference_writers(ref, fmt, case, tmp_path):
    film = _bad_films()[case]
    writer = (lambda p: ref.write_png(p, film, 0.0)) if fmt == crgpu.ENCODE_SRGB8 else (lambda p: ref.write_hdr(p, film))
    try:
        writer(tmp_path / "x")
        expected = None
    except ref.RefError as e:
        expected = str(e)
    try:
        oracle.encode(film, fmt)
        got = None
    except oracle.OracleError as e:
        got = str(e)
    assert got == expected


@pytest.mark.parametrize("exposure", [float("nan"), 100.5, -101.0])
def test_oracle_exposure_messages(ref, exposure, tmp_path):
    film = np.full((1, 2, 3), 0.5, np.float32)
    with pytest.raises(ref.RefError) as e1:
        ref.write_png(tmp_path / "x.png", film, exposure)
    with pytest.raises(oracle.OracleError) as e2:
        oracle.encode(film, crgpu.ENCODE_SRGB8, exposure)
    assert str(e1.value) == str(e2.value)
    with pytest.raises(crgpu.CrError) as e3:
        crgpu.display_thresholds(exposure)
    assert str(e3.value) == str(e1.value)


def _probe_values(table, rng):
    v = [np.float32(10.0) ** rng.uniform(-12, 12, size=200000).astype(np.float32),
         rng.uniform(0, 1, size=50000).astype(np.float32),
         np.array([0.0, -0.0, 1e-45, 1e-38, 0.0031308, 1.0, 2.0, FLT_MAX], np.float32)]
    finite = table[np.isfinite(table)]
    v += [finite, np.nextafter(finite, np.float32(0)), np.nextafter(finite, np.float32(np.inf))]
    return np.concatenate(v).astype(np.float32)


@pytest.mark.parametrize("exposure", [0.0, -2.0, 3.25, -24.0, 24.0, 100.0, -100.0, 0.7109375])
def test_display_threshold_table_equals_the_mapping(exposure):
    """The device encoder's byte is the largest k with table[k] <= value. The mapping is
    non-decreasing in the value (checked exhaustively over all non-negative floats at eight
    exposures when the table method was adopted), so the table reproduces it; here it is
    compared with direct evaluation at every threshold, its neighbours and 250k values."""
    t = crgpu.display_thresholds(exposure)
    assert t[0] == 0 and np.all(np.diff(t[np.isfinite(t)]) > 0)
    rng = np.random.default_rng(int(abs(exposure) * 1000) + 7)
    v = _probe_values(t, rng)
    v = v[np.isfinite(v)]
    v = np.concatenate([v, np.zeros((-len(v)) % 3072, np.float32)])
    direct = np.frombuffer(oracle.encode(v.reshape(-1, 1024, 3), crgpu.ENCODE_SRGB8, exposure), np.uint8)
    via_table = (np.searchsorted(t, v, side="right") - 1).astype(np.uint8)
    assert np.array_equal(direct, via_table)
