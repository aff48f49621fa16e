"""Build libgcz.so in-tree with nvcc for sm_100a.

    python gpu-compressor_b200/build.py [--force]

The library lands in gpu-compressor_b200/gcz/libgcz.so next to the Python
host package that loads it.  Rebuilds only when a source or header is newer.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(HERE, "gcz", "libgcz.so")

SOURCES = ["gcz_api.cu", "gcz_sweep.cu", "gcz_zstd.cu", "gcz_zstd2.cu", "gcz_lzma2.cu", "gcz_noalloc.cu", "gcz_gen.cpp",
           "gcz_frames.cpp", "gcz_zenc.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr"]


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def build(force=False, verbose=False):
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)
    ] + [os.path.abspath(__file__)]
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= _newest(deps):
        return OUT
    cmd = [NVCC] + ARCH + FLAGS + ["-I", INCLUDE, "-I", CSRC] + [os.path.join(CSRC, s) for s in SOURCES] + [
        "-o", OUT + ".tmp", "-lpthread", "-ldl"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
