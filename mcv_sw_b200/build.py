"""Builds libmcv_gpu.so in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libmcv_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

SOURCES = ["mcv_gpu.cu", "stage_d3_f64.cu", "stage_d3_mix.cu", "stage_d4_f64.cu", "stage_d4_mix.cu",
           "mcv_geometry.cu", "mcv_diag.cu", "mcv_noalloc.cu", "host_setup.cpp", "mcv_server.cpp"]
# per-source flags: the device geometry restates host formulas compiled
# without FMA contraction
SOURCE_FLAGS = {"mcv_geometry.cu": ["-fmad=false"]}
HEADERS = ["mcv_stage.cuh", "mcv_halo.cuh", "mcv_tma.cuh", "mcv_ksum.cuh", "mcv_internal.h", os.path.join("..", "..", "include", "mcv_gpu.h")]
OBJ_DIR = os.path.join(HERE, "_lib", "obj")

NVCC_FLAGS = [
    "-O3", "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off,-O2",
    "-ccbin", HOST_CXX,
]


def _stale():
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False, extra_flags=()):
    """Compile the CUDA/C++ library (one object per source, in parallel); returns its path."""
    if not force and not _stale():
        return LIB_PATH
    os.makedirs(OBJ_DIR, exist_ok=True)
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        cmd = [NVCC] + NVCC_FLAGS + SOURCE_FLAGS.get(src, []) + list(extra_flags) + ["-c", os.path.join(CSRC, src),
                                                                                    "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd)))
    failed = [src for src, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError(f"nvcc failed on {failed}")
    tmp = LIB_PATH + ".tmp"
    cmd = [NVCC, "-shared", "-ccbin", HOST_CXX, "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs + [
        "-lgomp"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra_flags=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
