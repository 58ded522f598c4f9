"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``spaqr_oracle.cpp`` into ``oracle/_build/libspaqr_oracle.so`` and links
it against the LAPACK/CBLAS exports of SciPy's bundled OpenBLAS
(``scipy_LAPACKE_*``, ``scipy_cblas_*``).  Only tests, ``__graft_entry__`` and the
CPU-baseline leg of ``bench.py`` use the result.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libspaqr_oracle.so")
SRC = os.path.join(HERE, "spaqr_oracle.cpp")


def openblas_path() -> str:
    import scipy

    libdir = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas*.so")))
    cands = [c for c in cands if "openblas64" not in os.path.basename(c)]
    if not cands:
        raise RuntimeError(f"SciPy's bundled OpenBLAS not found under {libdir}")
    return cands[0]


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    blas = openblas_path()
    cmd = [
        "g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", SRC, "-o", LIB,
        "-L" + os.path.dirname(blas), "-l:" + os.path.basename(blas),
        "-Wl,-rpath," + os.path.dirname(blas),
    ]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
