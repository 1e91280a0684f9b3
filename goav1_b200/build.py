"""Builds goav1_b200/libgoav1pf.so (the C-ABI library) with nvcc for sm_100a.

The library is built in-tree so it ships with the source tree; nothing is
installed.  Usage: python -m goav1_b200.build [--force]
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgoav1pf.so")
SOURCES = ["pf_api.cu", "pf_deblock.cu", "pf_cdef.cu", "pf_lr.cu", "pf_fg.cu", "pf_grain_static.cu", "pf_search.cu", "pf_mlp.cu", "pf_superres.cu",
           "pf_lfmask.cu", "pf_diag.cu"]
HEADERS = ["pf_common.cuh", "pf_cdef_dev.cuh", "pf_search.cuh", "pf_tables.h", os.path.join("..", "..", "include", "goav1pf.h")]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, h) for h in HEADERS]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [_nvcc()] + NVCC_FLAGS + inc + ["-dc" if False else "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs + ["-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print("built", LIB)
