"""Builds libpivb200.so (the CUDA path and its C ABI) in-tree for sm_100a with nvcc.

Translation units whose results must be bit-exact against the reference (placement, mask,
validation, preprocessing) are compiled with --fmad=false; the FFT correlation unit keeps FMA
contraction (it is checked to a tolerance).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpivb200.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", CSRC, "-I", os.path.join(ROOT, "include")]
UNITS = {
    "correlate.cu": [],
    "correlate_tc.cu": [],
    "field.cu": ["--fmad=false"],
    "prep.cu": ["--fmad=false"],
    "api.cu": ["--fmad=false"],
    "noalloc.cu": ["--fmad=false"],
    "post.cu": ["--fmad=false"],
}
HEADERS = ["common.cuh", "fft.cuh", "kernels.h", "window.cuh", "tc.cuh"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def build(force=False, verbose=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    nvcc = _nvcc()
    hdr_mtime = max(os.path.getmtime(os.path.join(CSRC, h)) for h in HEADERS)
    hdr_mtime = max(hdr_mtime, os.path.getmtime(os.path.join(ROOT, "include", "piv_b200.h")))
    objs = []
    rebuilt = False
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OUT_DIR, unit.replace(".cu", ".o"))
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime):
            continue
        cmd = [nvcc, *ARCH, *COMMON, *extra, "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        rebuilt = True
    if rebuilt or force or not os.path.exists(LIB):
        tmp = LIB + ".tmp"
        subprocess.run([nvcc, *ARCH, "-shared", *objs, "-o", tmp, "-lcudart"], check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
