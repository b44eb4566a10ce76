"""Builds the phx shared library (phenlei_b200/libphx.so) for sm_100a with nvcc.

    python -m phenlei_b200.build [--fmad=false]

The library is self-contained CUDA C++ behind the C ABI of include/phx.h; no
torch types cross it.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libphx.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["phx_kernels.cu", "phx_sa.cu", "phx_mlp.cu", "phx_noalloc.cu", "phx_halo.cu", "phx_host.cpp"]
# The face, gradient and SA passes of the FP32 working path use approximate
# single-precision division and square root (2 ulp); these flags leave FP64
# arithmetic alone.  At 16M cells: face pass 5.3 -> 4.3 ms, gradient 2.1 ->
# 1.8 ms.  The LU-SGS sweeps in the same files divide through idiv (IEEE).
FILE_FLAGS = {"phx_kernels.cu": ["-prec-div=false", "-prec-sqrt=false"],
              "phx_sa.cu": ["-prec-div=false", "-prec-sqrt=false"]}


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def needs_build(lib=LIB) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "phx.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(extra=(), lib=LIB, verbose=False) -> str:
    objs = []
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    common = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3", *ARCH, *extra]
    for src in SOURCES:
        obj = os.path.join(HERE, "_build", src + ".o")
        lang = ["-x", "cu"] if src.endswith(".cpp") else []
        cmd = [NVCC, *common, *FILE_FLAGS.get(src, ()), *lang, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = _run(cmd)
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    _run([NVCC, "-shared", *ARCH, *objs, "-o", lib, "-lcudart"])
    return lib


if __name__ == "__main__":
    extra = [a for a in sys.argv[1:] if a.startswith("--fmad")]
    print(build(extra=extra, verbose="-v" in sys.argv))
