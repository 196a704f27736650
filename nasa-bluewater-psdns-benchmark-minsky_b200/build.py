"""Build recipe for libpsdns_gpu.so (sm_100a).

Run as `python build.py` from anywhere; the shared library is written next to
this file so that it travels with the source tree.  Each translation unit is
compiled to an object under _build/ (in parallel, and only when it or a
header changed), then the objects are linked.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
UNITS = ("psdns_api.cu", "stage_noalloc.cu", "forcing.cpp", "tc_dft.cu", "learned.cu")
SRC = [os.path.join(CSRC, f) for f in UNITS if os.path.exists(os.path.join(CSRC, f))]
# psdns_api.cu is compiled once for the host code and once per grid size for
# that size's kernels (-DPSDNS_INST_N), so that the units build in parallel
GRID_SIZES = (16, 32, 48, 64, 96, 128, 256, 512, 1024)
JOBS = [(s, None) for s in SRC] + [(os.path.join(CSRC, "psdns_api.cu"), n) for n in GRID_SIZES]
OUT = os.path.join(HERE, "libpsdns_gpu.so")
OBJDIR = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++",
         "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return hs + [os.path.join(ROOT, "include", "psdns_gpu.h")]


def _obj(src, n=None):
    tag = "" if n is None else ".n%d" % n
    return os.path.join(OBJDIR, os.path.basename(src) + tag + ".o")


def _stale(target, deps):
    return not os.path.exists(target) or any(os.path.getmtime(target) < os.path.getmtime(d) for d in deps)


def build(verbose=False, extra=()):
    hdrs = _headers()
    if not extra and not _stale(OUT, SRC + hdrs):
        return OUT
    os.makedirs(OBJDIR, exist_ok=True)
    todo = [(s, n) for s, n in JOBS if extra or _stale(_obj(s, n), [s] + hdrs)]

    def compile_one(job):
        src, n = job
        defs = [] if n is None else ["-DPSDNS_INST_N=%d" % n]
        cmd = [NVCC] + FLAGS + defs + list(extra) + ["-c", "-o", _obj(src, n) + ".tmp", src]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(_obj(src, n) + ".tmp", _obj(src, n))

    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 4))) as ex:
        for f in [ex.submit(compile_one, j) for j in todo]:
            f.result()
    link = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-ccbin", "/usr/bin/g++",
            "-o", OUT + ".tmp"] + [_obj(s, n) for s, n in JOBS]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
