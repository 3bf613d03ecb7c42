"""Builds the in-tree CUDA library rapidsfm_b200/lib/librsfm_b200.so for sm_100a with nvcc.

Usage: python -m rapidsfm_b200.build   (or rapidsfm_b200.build.build_library()).
The build is incremental: it is skipped when the library is newer than every source file.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "librsfm_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = [
    "common.cu",
    "bf_match.cu",
    "bf_match_noalloc.cu",
    "bf_variants.cu",
    "filters.cu",
    "ransac.cu",
    "ranked_register.cpp",
    "precomp.cpp",
    "bf_autotune.cpp",
    "host_filters.cpp",
    "diag.cu",
    "cashash.cu",
    "cashash_match.cu",
    "cashash_ranked.cu",
    "mlp.cu",
]

# Compiled on their own with the reference's --use_fast_math (their float results must equal the
# reference's kernels', which are built with it), then linked with the rest.
FAST_MATH_SOURCES = [
    "cashash_bias_fastmath.cu",
]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _inputs():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(INCLUDE, "rsfm_b200.h"))
    return [f for f in files if os.path.isfile(f)]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _inputs())


def build_library(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = LIB + ".tmp"
    objs = []
    for s in FAST_MATH_SOURCES:
        obj = os.path.join(LIBDIR, os.path.splitext(s)[0] + ".o")
        flags = [f for f in NVCC_FLAGS if f != "-shared"]
        cmd = [_nvcc()] + flags + ["--use_fast_math", "-c", "-o", obj, os.path.join(CSRC, s)]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError(f"nvcc failed compiling {s}")
        objs.append(obj)
    cmd = [_nvcc()] + NVCC_FLAGS + ["-o", tmp] + [os.path.join(CSRC, s) for s in SOURCES] + objs
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building librsfm_b200.so")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose=True))
