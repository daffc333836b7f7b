"""The C-ABI library loads and exports every entry point include/cr_gpu.h declares, and
its GPU-free entry points behave like the reference (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def declared_functions():
    text = open(os.path.join(ROOT, "include", "cr_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(cr_[a-z0-9_]+)\s*\(", text))
    names.discard("cr_progress_fn")
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("cr_gpu_render", "cr_gpu_intersect", "cr_gpu_scene_create", "cr_bvh_build", "cr_scene_finalize"):
        assert required in names


def test_library_exports_every_declared_symbol(crgpu):
    out = subprocess.run(["nm", "-D", "--defined-only", crgpu.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if " T " in line)
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    lib = ctypes.CDLL(crgpu.LIB_PATH)
    for n in declared_functions():
        assert hasattr(lib, n)


def test_abi_version_and_no_device_is_not_an_error(crgpu):
    assert crgpu.lib.cr_gpu_abi_version() == 1
    assert crgpu.device_count() >= 0


def test_record_sizes_match_the_reference_types(crgpu):
    # cr::Triangle 188, cr::Ray 44, cr::Hit 32, Bvh::Node 32 (static_asserts in oracle/ref_shim.cpp)
    assert crgpu.triangle_dtype.itemsize == 188
    assert crgpu.ray_dtype.itemsize == 44
    assert crgpu.hit_dtype.itemsize == 32
    assert crgpu.node_dtype.itemsize == 32


@pytest.mark.parametrize("field,value,message", [
    ("width", 0, "Width and height must be in [1, 16384]"),
    ("height", 16385, "Width and height must be in [1, 16384]"),
    ("samples", 0, "Samples must be in [1, 1048576]"),
    ("samples", 1048577, "Samples must be in [1, 1048576]"),
    ("bounces", 65, "Bounces must be in [1, 64]"),
    ("threads", -1, "Threads must be 0 (automatic) or in [1, 256]"),
])
def test_options_validation_messages(crgpu, field, value, message):
    o = crgpu.Options.make()
    setattr(o, field, value)
    with pytest.raises(crgpu.CrError) as e:
        crgpu.validate_options(o)
    assert str(e.value) == message
    assert e.value.status == 1


def test_options_validation_matches_reference(crgpu, ref):
    cases = [dict(width=16384, height=4097), dict(width=16384, height=4096), dict(width=1, height=1, samples=1048576),
             dict(bounces=0), dict(threads=257), dict()]
    for c in cases:
        o = crgpu.Options.make(**c)
        try:
            ref.validate_options(o)
            expected = None
        except ref.RefError as e:
            expected = str(e)
        try:
            crgpu.validate_options(o)
            got = None
        except crgpu.CrError as e:
            got = str(e)
        assert got == expected, c


def test_environment_rotation_is_the_references(crgpu):
    # render.cpp:24: fmod(degrees, 360) * pi / 180 in float
    for deg in (0.0, 31.0, 90.0, 360.0, 725.5, -45.0):
        expected = np.float32(np.fmod(np.float32(deg), np.float32(360))) * np.float32(np.pi) / np.float32(180)
        assert crgpu.environment_rotation(deg) == pytest.approx(float(expected), rel=0, abs=0)
