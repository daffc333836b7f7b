"""Drop-in check: the reference's own integrator and transport-edge test suites
(tests/test_integrator.cpp, tests/test_transport_edges.cpp), compiled from its sources with
cr::render defined by cpu-renderer_b200/host/render_gpu.cpp (src/render.cpp compiled with
that function renamed, so cr::Environment is the reference's own), pass on the GPU backend.
The binaries are built by `make -f oracle/Makefile dropin` where the reference sources are
present and travel with the build tree."""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin")


@pytest.mark.parametrize("suite", ["integrator", "transport_edges"])
def test_reference_suite_on_gpu_backend(gpu, tmp_path, suite):
    exe = os.path.join(DROPIN, f"{suite}_tests")
    if not os.path.exists(exe):
        pytest.skip("drop-in test binaries not built (needs the reference sources)")
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=900)
    print(r.stdout[-3000:])
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
