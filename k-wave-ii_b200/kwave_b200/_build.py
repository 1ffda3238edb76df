"""Build recipe of the in-tree CUDA library (sm_100a only).

``build()`` compiles the library's translation units in parallel and links
libkwave_b200.so next to this file, so the built library travels with the
source tree:

* csrc/kwave_b200.cu -- host side, C ABI, auxiliary kernels;
* csrc/kw_inst.cu, once per compile-time axis length (-DKW_INST_N=<n>) and
  once for the runtime-radix kernels (-DKW_INST_N=0): the transform and
  stage kernels and their launchers.

Objects go to csrc/_build/ (git-ignored).
"""
from __future__ import annotations

import concurrent.futures
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "csrc")
OBJ = os.path.join(CSRC, "_build")
OUT = os.path.join(HERE, "libkwave_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]
# compile-time axis lengths (KW_STATIC_SIZES in csrc/kw_plan.cuh) and 0 for
# the runtime-radix kernels
INST_SIZES = (0, 64, 96, 128, 160, 192, 256, 320, 384, 512)


def sources():
    d = CSRC
    return [os.path.join(d, f) for f in sorted(os.listdir(d)) if f.endswith((".cu", ".cuh", ".inc"))] + \
        [os.path.join(os.path.dirname(ROOT), "include", "kwave_b200.h")]


def units():
    """(source, extra flags, object) of every translation unit."""
    u = [(os.path.join(CSRC, "kwave_b200.cu"), [], os.path.join(OBJ, "kwave_b200.o"))]
    for n in INST_SIZES:
        u.append((os.path.join(CSRC, "kw_inst.cu"), ["-DKW_INST_N=%d" % n], os.path.join(OBJ, "kw_inst_%d.o" % n)))
    return u


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force=False, verbose=False, jobs=None):
    if not force and up_to_date():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose else []

    def compile_one(unit):
        src, flags, obj = unit
        cmd = [nvcc] + NVCC_FLAGS + extra + flags + ["-c", "-o", obj, src]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    jobs = jobs or max(1, min(len(INST_SIZES) + 1, os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(compile_one, units()))
    for cmd, r in results:
        if verbose or r.returncode:
            print(" ".join(cmd))
            print(r.stdout + r.stderr)
        if r.returncode:
            raise subprocess.CalledProcessError(r.returncode, cmd, r.stdout, r.stderr)
    cmd = [nvcc] + ARCH + ["-shared", "-o", OUT] + [u[2] for u in units()]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force=True, verbose=True)
