"""Build recipe for libpsdns_gpu.so (sm_100a).

Run as `python build.py` from anywhere; the shared library is written next to
this file so that it travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = [os.path.join(HERE, "csrc", f) for f in ("psdns_api.cu", "stage_noalloc.cu", "forcing.cpp")]
OUT = os.path.join(HERE, "libpsdns_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def build(verbose=False, extra=()):
    deps = SRC + [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))]
    deps.append(os.path.join(ROOT, "include", "psdns_gpu.h"))
    if os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(d) for d in deps) and not extra:
        return OUT
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
           "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-shared", "-ccbin", "/usr/bin/g++",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(HERE, "csrc"),
           "-o", OUT + ".tmp"] + list(extra) + SRC
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
