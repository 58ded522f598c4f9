"""ctypes wrapper of the CPU oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, always as the checker or the timed CPU
baseline; the product package never does.  The oracle restates the reference
ParTree in sequential C++ on LAPACK (see ``spaqr_oracle.cpp``); parity is
unpinned because the reference itself cannot be built or run here.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build_oracle

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build_oracle.LIB
        if not os.path.exists(path):
            path = build_oracle.build()
        L = C.CDLL(path)
        vp, i32, f64 = C.c_void_p, C.c_int, C.c_double
        pi, pd = C.POINTER(C.c_int), C.POINTER(C.c_double)
        sig = {
            "orc_create": (vp, [i32, i32, f64, i32]),
            "orc_destroy": (None, [vp]),
            "orc_set_threads": (i32, [vp, i32]),
            "orc_set_pivot": (i32, [vp, i32, f64]),
            "orc_set_matrix": (i32, [vp, i32, i32, pi, pi, pd, i32]),
            "orc_get_matrix_values": (i32, [vp, pd]),
            "orc_set_coords_tensor": (i32, [vp, i32, i32]),
            "orc_partition": (i32, [vp]),
            "orc_assemble": (i32, [vp]),
            "orc_factorize": (i32, [vp]),
            "orc_solve_inplace": (i32, [vp, pd]),
            "orc_solve_global": (i32, [vp, pd, pd]),
            "orc_spmv": (i32, [vp, pd, pd]),
            "orc_gmres": (i32, [vp, pd, i32, f64, pi, pd, pd, i32]),
            "orc_n": (i32, [vp]),
            "orc_get_perm": (i32, [vp, pi]),
            "orc_num_clusters": (i32, [vp]),
            "orc_level_count": (i32, [vp, i32, i32]),
            "orc_level_first": (i32, [vp, i32]),
            "orc_cluster_info": (i32, [vp, i32, pi]),
            "orc_num_edges": (i32, [vp]),
            "orc_block_shape": (i32, [vp, i32, i32, pi]),
            "orc_block": (i32, [vp, i32, i32, pd]),
            "orc_edges": (i32, [vp, pi]),
            "orc_qsp_shape": (i32, [vp, i32, pi]),
            "orc_qsp": (i32, [vp, i32, pd, pd]),
            "orc_time": (f64, [vp, i32]),
            "orc_random_reference": (i32, [i32, i32, pd]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _pi(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _pd(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


INFO_FIELDS = ("lvl", "merge_lvl", "rows", "cols", "rank", "parent", "cstart", "sep", "l_lvl", "l_sep",
               "r_lvl", "r_sep", "section", "cols_org", "sparsified", "nchildren")


def random_reference(n: int, seed: int) -> np.ndarray:
    """The reference's RHS generator (util.cpp:992-1001): mt19937 + U(-1, 1)."""
    out = np.empty(n)
    lib().orc_random_reference(n, seed, _pd(out))
    return out


class OracleTree:
    """Sequential CPU restatement of ParTree (square systems, tensor-grid ordering)."""

    def __init__(self, nlevels: int, skip: int = 0, tol: float = 1e-1, nthreads: int = 1):
        self.h = lib().orc_create(nlevels, skip, tol, nthreads)
        if not self.h:
            raise ValueError("oracle: bad parameters")
        self.nlevels = nlevels

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def _chk(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"oracle {what} failed with status {rc}")

    def set_pivot(self, mode: int, rtol: float = 1e-6):
        """mode 1 (default): restated dlaqp2, pivot = first column within rtol of the
        largest partial norm; mode 0: LAPACK dgeqp3 exactly as the reference calls it."""
        lib().orc_set_pivot(self.h, mode, rtol)

    def set_threads(self, t: int):
        lib().orc_set_threads(self.h, t)

    def set_matrix(self, colptr, rowidx, vals, scale: bool = True):
        colptr = np.ascontiguousarray(colptr, dtype=np.int32)
        rowidx = np.ascontiguousarray(rowidx, dtype=np.int32)
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        self.n = len(colptr) - 1
        self.nnz = int(colptr[-1])
        self._chk(lib().orc_set_matrix(self.h, self.n, self.n, _pi(colptr), _pi(rowidx), _pd(vals), int(scale)),
                  "set_matrix")

    def matrix_values(self):
        out = np.empty(self.nnz)
        lib().orc_get_matrix_values(self.h, _pd(out))
        return out

    def set_coords_tensor(self, n: int, d: int):
        self._chk(lib().orc_set_coords_tensor(self.h, n, d), "set_coords")

    def partition(self):
        self._chk(lib().orc_partition(self.h), "partition")

    def assemble(self):
        self._chk(lib().orc_assemble(self.h), "assemble")

    def factorize(self):
        self._chk(lib().orc_factorize(self.h), "factorize")

    def solve_inplace(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        self._chk(lib().orc_solve_inplace(self.h, _pd(x)), "solve")
        return x

    def solve_global(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        self._chk(lib().orc_solve_global(self.h, _pd(b), _pd(x)), "solve_global")
        return x

    def spmv(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        self._chk(lib().orc_spmv(self.h, _pd(x), _pd(y)), "spmv")
        return y

    def gmres(self, b, maxit: int = 300, tol: float = 1e-12):
        x = np.ascontiguousarray(b, dtype=np.float64).copy()
        iters = C.c_int(0)
        relres = C.c_double(0)
        hist = np.zeros(maxit)
        self._chk(lib().orc_gmres(self.h, _pd(x), maxit, tol, C.byref(iters), C.byref(relres), _pd(hist), maxit),
                  "gmres")
        return x, iters.value, relres.value, hist[: iters.value + 1].copy()

    def perm(self):
        p = np.empty(self.n, dtype=np.int32)
        lib().orc_get_perm(self.h, _pi(p))
        return p

    def num_clusters(self):
        return lib().orc_num_clusters(self.h)

    def level(self, lvl: int):
        """Cluster orders at level ``lvl``: (all, interiors count, interfaces count)."""
        first = lib().orc_level_first(self.h, lvl)
        cnt = lib().orc_level_count(self.h, lvl, 0)
        return list(range(first, first + cnt)), lib().orc_level_count(self.h, lvl, 1), lib().orc_level_count(self.h, lvl, 2)

    def cluster(self, order: int) -> dict:
        info = np.zeros(16, dtype=np.int32)
        self._chk(lib().orc_cluster_info(self.h, order, _pi(info)), "cluster_info")
        return dict(zip(INFO_FIELDS, info.tolist()))

    def clusters(self):
        return [self.cluster(o) for o in range(self.num_clusters())]

    def edges(self):
        m = lib().orc_num_edges(self.h)
        out = np.zeros(4 * m, dtype=np.int32)
        lib().orc_edges(self.h, _pi(out))
        return out.reshape(m, 4)

    def block(self, n1: int, n2: int):
        shape = np.zeros(2, dtype=np.int32)
        if lib().orc_block_shape(self.h, n1, n2, _pi(shape)) != 0:
            return None
        out = np.zeros(int(shape[0]) * int(shape[1]))
        lib().orc_block(self.h, n1, n2, _pd(out))
        return out.reshape(int(shape[1]), int(shape[0])).T

    def qsp(self, order: int):
        shape = np.zeros(2, dtype=np.int32)
        lib().orc_qsp_shape(self.h, order, _pi(shape))
        V = np.zeros(int(shape[0]) * int(shape[1]))
        tau = np.zeros(int(shape[1]))
        lib().orc_qsp(self.h, order, _pd(V), _pd(tau))
        return V.reshape(int(shape[1]), int(shape[0])).T, tau

    def times(self):
        return {k: lib().orc_time(self.h, i) for i, k in enumerate(("partition", "assemble", "factorize", "solve", "gmres"))}
