"""Builds libcr_b200.so, the sm_100a path tracer behind include/cr_gpu.h.

The CUDA translation unit is compiled with --fmad=false: the device code restates the
reference's float/double expressions and must round each operation separately, as the
reference does on x86-64 without FMA. The host preparation code (cr_host.cpp) is compiled
by g++ with the reference's own Release flags so its tables match bit for bit.

Usage: python cpu-renderer_b200/build.py [--force] [--verbose]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcr_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC",
              "-Xptxas", "-warn-spills", "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O3", "-DNDEBUG", "-std=c++17", "-fPIC", "-pthread"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("command failed: " + " ".join(cmd))
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)
    return r


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))] + [os.path.join(INCLUDE, "cr_gpu.h"), __file__]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in _sources())


def build(force=False, verbose=False, ptxas_verbose=False, defines=(), out=None):
    """Compile the library in-tree (or to `out` with extra -D defines); returns its path."""
    lib = out or LIB
    if not force and not defines and out is None and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    inc = ["-I" + INCLUDE, "-I" + CSRC]
    tag = "" if out is None else "_" + os.path.basename(out).replace(".so", "")
    host_obj = os.path.join(BUILD, "cr_host.o")
    _run(["g++"] + CXX_FLAGS + inc + ["-I/usr/local/cuda/include", "-c", os.path.join(CSRC, "cr_host.cpp"), "-o", host_obj], verbose)
    flags = NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_verbose else []) + ["-D" + d for d in defines]
    dev_objs, jobs = [], []
    for cu in sorted(f for f in os.listdir(CSRC) if f.endswith(".cu")):
        obj = os.path.join(BUILD, cu[:-3] + tag + ".o")
        cmd = [nvcc] + ARCH + flags + inc + ["-c", os.path.join(CSRC, cu), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        jobs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        dev_objs.append(obj)
    failed = None
    for cmd, proc in jobs:  # the translation units compile in parallel
        out, err = proc.communicate()
        if proc.returncode != 0:
            sys.stderr.write(out + err)
            failed = cmd
        elif ptxas_verbose or (verbose and (out or err)):
            sys.stderr.write(out + err)
    if failed:
        raise RuntimeError("command failed: " + " ".join(failed))
    tmp = lib + ".tmp"
    _run([nvcc] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", tmp] + dev_objs + [host_obj, "-lpthread"], verbose)
    os.replace(tmp, lib)
    if tag:  # a variant build's objects are not reused: do not let them pile up in _build
        for obj in dev_objs:
            os.remove(obj)
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv, ptxas_verbose="--ptxas" in sys.argv)
    print(LIB)
