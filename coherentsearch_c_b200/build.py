"""In-tree build of the native libraries (sm_100a).

    python -m coherentsearch_c_b200.build

produces, under coherentsearch_c_b200/lib/:
  libcsgpu.so            CUDA backend: the reference's cs_gpu_* ABI plus
                         cs_b200.h (self-contained; host helpers hidden)
  libcoherent_search.so  host C: planning, search_file, candidates, .cohout
The command-line drivers are the reference's own (src/CoherentSearch.c,
src/list_main.c) linked against these libraries; oracle/Makefile's `dropin`
target builds them that way for the tests.
Compiled with nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo; host C
with -ffp-contract=off (the reference's FP contract, src/Makefile:43).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(CSRC, "host")
LIB = os.path.join(PKG, "lib")
OBJ = os.path.join(ROOT, "_build", "obj")
INC = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O2", "-fPIC", "-std=gnu11", "-ffp-contract=off", "-Wall", "-Wextra",
          "-Wno-unused-parameter", "-Wno-sign-compare", f"-I{INC}", f"-I{CSRC}"]

HOST_COMMON = ["cs_common.c"]
HOST_GPU_ONLY = ["cs_tables.c"]
HOST_LIB = ["cs_common.c", "cs_search.c"]
CUDA_SRCS = ["cs_gpu.cu", "cs_dedisp.cu", "cs_spectrum.cu", "cs_ducy.cu",
             "cs_collapse.cu", "cs_clip.cu"]
# FP64 candidate arithmetic that must round like the host restatements, which
# are built with -ffp-contract=off: no multiply-add contraction
CUDA_FLAGS = {"cs_ducy.cu": ["-fmad=false"], "cs_collapse.cu": ["-fmad=false"],
              "cs_clip.cu": ["-fmad=false"]}


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)
    return r


def _newer(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(INC, f) for f in os.listdir(INC) if f.endswith(".h")]
    hs += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs


def build(verbose: bool = False, force: bool = False) -> None:
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    hdrs = _headers()

    # host C for the GPU library, helpers hidden
    gpu_objs = []
    for src in HOST_COMMON + HOST_GPU_ONLY:
        s = os.path.join(HOST, src)
        o = os.path.join(OBJ, "gpu_" + src.replace(".c", ".o"))
        if force or _newer(o, [s] + hdrs):
            _run(["gcc"] + CFLAGS + ["-DCS_HIDDEN", "-fvisibility=hidden", "-c", s, "-o", o],
                 verbose)
        gpu_objs.append(o)
    for src in CUDA_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        if force or _newer(o, [s] + hdrs):
            _run([NVCC] + GENCODE + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler",
                  "-fPIC,-fvisibility=hidden", f"-I{INC}", f"-I{CSRC}"] +
                 CUDA_FLAGS.get(src, []) + ["-c", s, "-o", o], verbose)
        gpu_objs.append(o)
    libgpu = os.path.join(LIB, "libcsgpu.so")
    if force or _newer(libgpu, gpu_objs):
        cudalib = os.path.join(os.path.dirname(os.path.dirname(NVCC)), "lib64")
        _run([NVCC] + GENCODE + ["-shared", "-o", libgpu] + gpu_objs +
             [f"-L{cudalib}", "-lcufft", "-Xlinker", f"-rpath={cudalib}"], verbose)

    # host library (exports the coherent_search.h host API)
    host_objs = []
    for src in HOST_LIB:
        s = os.path.join(HOST, src)
        o = os.path.join(OBJ, "host_" + src.replace(".c", ".o"))
        if force or _newer(o, [s] + hdrs):
            _run(["gcc"] + CFLAGS + ["-c", s, "-o", o], verbose)
        host_objs.append(o)
    libhost = os.path.join(LIB, "libcoherent_search.so")
    if force or _newer(libhost, host_objs + [libgpu]):
        _run(["gcc", "-shared", "-o", libhost] + host_objs +
             [f"-L{LIB}", "-lcsgpu", "-Wl,-rpath,$ORIGIN", "-lm"], verbose)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print("built", LIB)
