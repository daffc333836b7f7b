"""Device allocation failures leave the library usable.

The reference reports a failed allocation as an exception and leaves its objects as they were.
Here `cr_gpu_debug_fail_allocation(n)` makes the nth device allocation from now fail as out of
memory (a host-side injection: the allocator throws before asking the driver, and every
allocation of a scene upload or a render comes before that call launches any kernel). For each
allocation of a scene upload, and of renders that grow the render workspace, the film and the
alias tables, the failing call must return CR_ERR_OUT_OF_MEMORY; the last film must then be
either a completed render's or absent; and the same calls made again after disarming must
render films bit-identical to those of scenes that never saw a failure. The scenario runs in a
child process, so the workspace starts empty and an armed injection cannot reach other tests.
"""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

CHILD = r"""
import json, sys
import numpy as np
import crgpu, workloads

OK, INVALID, OOM = 0, 1, 6
sc = workloads.sunlit_room_scene()
sky = workloads.sky_image(width=128, height=64)
tris, _ = crgpu.finalize(sc["triangles"], sc["materials"])
mats, cam = sc["materials"], sc["camera"]
alias = crgpu.Tuning()
alias.env_alias = 1

def scene():
    return crgpu.GpuScene(tris, mats, env=crgpu.env_desc(image=sky))

def opts(k):  # 1024 + 128 k samples: every k needs a larger pool, chunk and film than k - 1
    return crgpu.Options.make(width=32 + 4 * k, height=16, samples=2, bounces=4, seed=42)

def injected(e):
    assert e.status == OOM and "injected failure" in str(e), (e.status, str(e))

report = {"create_failures": 0, "render_failures": 0, "encode_after_failure": {}}

# every allocation of a scene upload (the environment tables are built on a helper thread)
n = 0
while True:
    crgpu.fail_allocation(n)
    try:
        g = scene()
    except crgpu.CrError as e:
        injected(e)
        crgpu.fail_allocation(-1)
        report["create_failures"] += 1
        n += 1
        assert n < 400, "scene upload never completed"
        continue
    crgpu.fail_allocation(-1)
    g.close()
    break

# every allocation of two renders (CDF then alias sampling) on a fresh scene with a small film
recovered = {}
k, quiet = 1, 0
while quiet < 2:
    g = scene()
    small = crgpu.Options.make(width=8, height=8, samples=1, bounces=4, seed=42)
    g.render(cam, small)
    big = opts(k)
    crgpu.fail_allocation(k - 1)
    failed = False
    try:
        g.render(cam, big)
        g.render(cam, big, tuning=alias)
    except crgpu.CrError as e:
        injected(e)
        failed = True
    crgpu.fail_allocation(-1)
    report["render_failures"] += int(failed)
    quiet = 0 if failed else quiet + 1
    # the last film is a completed render's (the small one or the big one) or there is none
    try:
        b = g.film_encode()
        assert len(b) in (3 * 8 * 8, 3 * big.width * big.height), len(b)
        report["encode_after_failure"][str(k)] = len(b)
    except crgpu.CrError as e:
        assert e.status == INVALID and "render first" in str(e), (e.status, str(e))
        report["encode_after_failure"][str(k)] = "no film"
    recovered[k] = (g.render(cam, big)[0], g.render(cam, big, tuning=alias)[0])
    g.close()
    k += 1
    assert k < 400, "renders never completed"

# the same renders in scenes that never saw a failure
mismatch = []
for k, (cdf, ali) in recovered.items():
    g = scene()
    a = g.render(cam, opts(k))[0]
    b = g.render(cam, opts(k), tuning=alias)[0]
    g.close()
    if a.tobytes() != cdf.tobytes() or b.tobytes() != ali.tobytes():
        mismatch.append(k)
report["sizes"] = len(recovered)
report["mismatch"] = mismatch
print("REPORT " + json.dumps(report))
"""


@pytest.mark.gpu
def test_allocation_failures_leave_scenes_and_renders_usable(gpu):
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([os.path.join(ROOT, "cpu-renderer_b200"), env.get("PYTHONPATH", "")])
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("REPORT ")][-1]
    report = json.loads(line[len("REPORT "):])
    # a scene upload makes well over ten device allocations, two renders that grow the
    # workspace, film and alias tables over thirty: each one failed once
    assert report["create_failures"] >= 10, report
    assert report["render_failures"] >= 30, report
    assert report["mismatch"] == [], report
    assert "no film" in report["encode_after_failure"].values(), report
