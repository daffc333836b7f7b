"""The drop-in library's composition (no GPU needed).

oracle/Makefile builds the reference's renderer library with cpu-renderer_b200/host/
render_gpu.cpp added and src/render.cpp compiled under -Drender=cr_reference_cpu_render.
Exactly one object may then define cr::render (ours), while cr::Environment and
RenderOptions::validate come from the reference's own render.cpp (render.cpp:12-104), not
from a restatement in the drop-in.
"""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

OBJ = os.path.join(ROOT, "oracle", "_ref", "dropin", "obj")


def defined(obj):
    out = subprocess.run(["nm", "-C", "--defined-only", obj], capture_output=True, text=True, check=True).stdout
    return {line.split(" ", 2)[2] for line in out.splitlines() if line.count(" ") >= 2 and line.split(" ")[1] in "TW"}


@pytest.mark.skipif(not os.path.isdir(OBJ) or shutil.which("nm") is None,
                    reason="drop-in objects are built only where the reference sources are present")
def test_only_render_is_ours():
    ours = defined(os.path.join(OBJ, "render_gpu.o"))
    theirs = defined(os.path.join(OBJ, "render_reference.o"))
    render = [s for s in ours if s.startswith("cr::render(")]
    assert len(render) == 1, ours
    assert not any(s.startswith("cr::render(") for s in theirs), "the reference's render was not renamed"
    assert any(s.startswith("cr::cr_reference_cpu_render(") for s in theirs)
    for member in ("cr::Environment::Environment(", "cr::Environment::sample(", "cr::Environment::pdf(",
                   "cr::Environment::radiance(", "cr::RenderOptions::validate("):
        assert any(s.startswith(member) for s in theirs), member
        assert not any(s.startswith(member) for s in ours), member
