"""Build the sm_100a shared library ``libspaqr_b200.so`` (and the ``spaqr`` driver).

The library is compiled in-tree with nvcc for ``sm_100a`` only; it holds the
host-side partition/symbolic code, the device engine and all CUDA kernels,
behind the C ABI declared in ``include/spaqr_b200.h``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libspaqr_b200.so")
DRIVER = os.path.join(HERE, "spaqr")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["structure.cpp", "engine.cu", "kernels.cu", "learned.cu", "noalloc.cu", "shard.cpp", "capi.cpp", "capi_learned.cpp"]
HEADERS = ["structure.hpp", "engine.hpp", "tasks.hpp", "kernels.hpp", "dense.cuh", "tc_apply.cuh", "noalloc.hpp", "learned.hpp",
           "capi_internal.hpp", "shard.hpp"]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "spaqr_b200.h")]
    if force or _stale(LIB, deps):
        objdir = os.path.join(HERE, "_build")
        os.makedirs(objdir, exist_ok=True)
        objs = []
        for src in SOURCES:
            obj = os.path.join(objdir, src + ".o")
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-c",
                   os.path.join(CSRC, src), "-o", obj]
            if src.endswith(".cu"):
                cmd.insert(1, "-Xptxas=-v" if verbose else "-Xptxas=-O3")
            subprocess.run(cmd, check=True)
            objs.append(obj)
        subprocess.run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"], check=True)
    drv_src = os.path.join(CSRC, "driver.cpp")
    if os.path.exists(drv_src) and (force or _stale(DRIVER, [drv_src, LIB])):
        subprocess.run(["g++", "-O2", "-std=c++17", drv_src, "-o", DRIVER, "-I" + os.path.join(ROOT, "include"),
                        "-L" + HERE, "-lspaqr_b200", "-Wl,-rpath,$ORIGIN"], check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
