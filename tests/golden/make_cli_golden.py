"""Golden outputs of the reference's own command-line renderer on its bundled harbor scene.

Needs `make -f oracle/Makefile cli data` (the reference CLI built from its sources into
oracle/_ref/cli/cpu_renderer and the harbor scene copied to oracle/_ref/data):

    python tests/golden/make_cli_golden.py

Writes harbor_cli_192x108_16spp.{png,hdr,txt}: the CLI's PNG, its linear RGBE .hdr and its
report lines, for the arguments in HARBOR_ARGS. tests/test_gpu_cli.py runs the same command
line through the drop-in GPU build of the same CLI and compares. Also writes
harbor_benchmark_cpu.txt, the report of the reference's phase benchmark (tests/benchmark.cpp)
on the same scene, which tests/test_gpu_phases.py compares with the GPU drop-in's.
"""
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DATA = os.path.join(ROOT, "oracle", "_ref", "data")
CPU_CLI = os.path.join(ROOT, "oracle", "_ref", "cli", "cpu_renderer")
CPU_BENCH = os.path.join(ROOT, "oracle", "_ref", "cli", "renderer_benchmark")
BENCH_NAME = "harbor_benchmark_cpu.txt"


def benchmark_command(program):
    return [program, os.path.join(DATA, "scenes", "harbor", "harbor.glb"), os.path.join(DATA, "scenes", "harbor", "sky.hdr")]
NAME = "harbor_cli_192x108_16spp"
HARBOR_ARGS = ["--width", "192", "--height", "108", "--samples", "16", "--bounces", "8", "--seed", "42"]


def harbor_command(cli, out_png):
    return [cli, "--scene", os.path.join(DATA, "scenes", "harbor", "harbor.glb"),
            "--environment", os.path.join(DATA, "scenes", "harbor", "sky.hdr"), *HARBOR_ARGS, "--output", out_png]


def main():
    if not os.path.exists(CPU_CLI):
        sys.exit("build the reference CLI first: make -f oracle/Makefile cli data")
    with tempfile.TemporaryDirectory() as tmp:
        png = os.path.join(tmp, NAME + ".png")
        r = subprocess.run(harbor_command(CPU_CLI, png) + ["--threads", str(os.cpu_count())],
                           capture_output=True, text=True, check=True)
        shutil.copy(png, os.path.join(HERE, NAME + ".png"))
        shutil.copy(png[:-4] + ".hdr", os.path.join(HERE, NAME + ".hdr"))
        with open(os.path.join(HERE, NAME + ".txt"), "w") as f:
            f.write(r.stdout.replace(tmp + os.sep, "").replace(DATA + os.sep, ""))
    print(r.stdout)
    b = subprocess.run(benchmark_command(CPU_BENCH), capture_output=True, text=True, check=True)
    with open(os.path.join(HERE, BENCH_NAME), "w") as f:
        f.write(b.stdout)
    print(b.stdout)


if __name__ == "__main__":
    main()
