"""Build librso.so (the CUDA library behind include/rso.h) for sm_100a.

Each translation unit under csrc/ is compiled with nvcc into _build/ and the
objects are linked into robustoptspline3d_b200/librso.so in-tree.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librso.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xcompiler", "-Wno-unused-function", "-ccbin", "g++"]

# voxelize.cu and boundary.cu round every operation separately, as their host
# restatements do (no fused multiply-add contraction)
FILE_FLAGS = {"voxelize.cu": ["-fmad=false"], "boundary.cu": ["-fmad=false"]}

SOURCES = ["capi.cu", "topology.cu", "fine_op.cu", "coarse_op.cu", "reduce.cu", "solver.cu", "design.cu",
           "design_capi.cu", "worst.cu", "mma.cu", "driver.cu", "prof.cu",
           "filter_noalloc.cu", "batch.cu", "autotune.cu", "oc.cu", "voxelize.cu",
           "boundary.cu", "dense.cu", "rigid.cu", "surface.cu"]


def _compile(src, verbose=False):
    obj = os.path.join(OUT_DIR, os.path.splitext(src)[0] + ".o")
    path = os.path.join(SRC, src)
    deps = [path, os.path.join(SRC, "rso_internal.cuh"), os.path.join(HERE, "..", "include", "rso.h")]
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj, None
    cmd = [NVCC] + ARCH + FLAGS + FILE_FLAGS.get(src, []) + ["-c", path, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stderr + r.stdout
    if verbose:
        sys.stderr.write(r.stderr)
    return obj, None


def build(verbose=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr + r.stdout)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
