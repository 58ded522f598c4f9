"""Python mirror of the reference ParTree API over the C ABI (ctypes).

``ParTree`` keeps the reference's call sequence and setter names
(ptree.h:122-160, tree.h:299-305): construct with ``(nlevels, skip)``, set
options, ``partition(A)`` -> ``assemble(A)`` -> ``factorize()`` ->
``solve(...)``; ``dist_gmres`` mirrors is.cpp:447-527.  All numerics run in
``libspaqr_b200.so`` on the GPU; there is no CPU fallback -- a missing or
unloadable library raises.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libspaqr_b200.so")
_lib = None


class SpqError(RuntimeError):
    def __init__(self, what: str, status: int, msg: str):
        super().__init__(f"{what} failed (status {status}): {msg}")
        self.status = status


def lib():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m pspaqr_public_b200.build` first")
        L = C.CDLL(LIB_PATH)
        vp, i32, f64, f32 = C.c_void_p, C.c_int, C.c_double, C.c_float
        pi, pd, pf = C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_float)
        sig = {
            "spq_create": (i32, [i32, i32, C.POINTER(vp)]),
            "spq_destroy": (i32, [vp]),
            "spq_set_tol": (i32, [vp, f64]),
            "spq_set_skip": (i32, [vp, i32]),
            "spq_set_scale": (i32, [vp, i32]),
            "spq_set_order": (i32, [vp, f32]),
            "spq_set_hsl": (i32, [vp, i32]),
            "spq_set_nthreads": (i32, [vp, i32]),
            "spq_set_verbose": (i32, [vp, i32]),
            "spq_set_ttor_log": (i32, [vp, i32]),
            "spq_set_square": (i32, [vp, i32]),
            "spq_set_pivot_rtol": (i32, [vp, f64]),
            "spq_set_rrqr_work": (i32, [vp, f64, f64]),
            "spq_set_precision": (i32, [vp, i32]),
            "spq_set_krylov": (i32, [vp, i32]),
            "spq_set_tensor_cores": (i32, [vp, i32]),
            "spq_tune_table": (i32, [vp, pf]),
            "spq_set_spin_limit": (i32, [vp, C.c_longlong]),
            "spq_set_checks": (i32, [vp, i32]),
            "spq_set_plan_cache": (i32, [vp, i32]),
            "spq_plan_hits": (C.c_longlong, [vp]),
            "spq_debug_corrupt_descriptor": (i32, [vp]),
            "spq_get_factor": (i32, [vp, i32, i32, pd, pi]),
            "spq_set_coords": (i32, [vp, i32, i32, pd]),
            "spq_set_coords_tensor": (i32, [vp, i32, i32]),
            "spq_partition": (i32, [vp, i32, i32, pi, pi, pd]),
            "spq_assemble": (i32, [vp]),
            "spq_factorize": (i32, [vp]),
            "spq_solve_inplace": (i32, [vp, pd]),
            "spq_solve_inplace_device": (i32, [vp, vp]),
            "spq_solve_global": (i32, [vp, pd, pd]),
            "spq_spmv": (i32, [vp, pd, pd]),
            "spq_factor_backward_error": (i32, [vp, i32, pd, C.c_ulonglong, pd]),
            "spq_gmres": (i32, [vp, pd, i32, f64, pi, pd, pd, i32]),
            "spq_gmres_device": (i32, [vp, vp, i32, f64, pi, pd, pd, i32]),
            "spq_gmres_device_noalloc": (i32, [vp, vp, i32, f64, pi, pd]),
            "spq_rank_model_size": (i32, [pi, pi]),
            "spq_set_rank_model": (i32, [vp, pf, pf, pf, i32]),
            "spq_learned_counts": (i32, [vp, C.POINTER(C.c_longlong)]),
            "spq_set_sketch_tuning": (i32, [vp, f64, i32]),
            "spq_set_rank_margin": (i32, [vp, f32]),
            "spq_set_rank_log": (i32, [vp, i32]),
            "spq_rank_log_count": (i32, [vp]),
            "spq_rank_log": (i32, [vp, pf, pi, pi, pi]),
            "spq_rank_log_clear": (i32, [vp]),
            "spq_mlp_loss_grad": (i32, [pf, pf, pf, i32, pf, pf]),
            "spq_mlp_predict": (i32, [pf, pf, i32, pf]),
            "spq_mlp_train": (i32, [pf, pf, pf, i32, i32, i32, f32, C.c_ulonglong, pf]),
            "spq_mlp_last_error": (C.c_char_p, []),
            "spq_distribute_x": (i32, [vp, pd, pd]),
            "spq_solve_block_device": (i32, [vp, vp, i32, C.c_longlong]),
            "spq_gmres_block": (i32, [vp, pd, i32, C.c_longlong, i32, f64, pi, pd]),
            "spq_gmres_block_device": (i32, [vp, vp, i32, C.c_longlong, i32, f64, pi, pd]),
            "spq_extract_x": (i32, [vp, pd, pd]),
            "spq_n": (i32, [vp]),
            "spq_set_stream": (i32, [vp, vp]),
            "spq_scale_columns": (i32, [i32, pi, pd]),
            "spq_random_reference": (i32, [i32, i32, pd]),
            "spq_get_perm": (i32, [vp, pi]),
            "spq_num_clusters": (i32, [vp]),
            "spq_num_levels": (i32, [vp]),
            "spq_cluster_info": (i32, [vp, i32, pi]),
            "spq_level_range": (i32, [vp, i32, pi, pi]),
            "spq_num_edges": (i32, [vp]),
            "spq_find_edge": (i32, [vp, i32, i32]),
            "spq_get_block": (i32, [vp, i32, i32, pd, pi]),
            "spq_shard_plan": (i32, [vp, i32, pi, pi, pi]),
            "spq_shard_exchange": (i32, [vp, i32, i32, pi]),
            "spq_get_edges": (i32, [vp, pi]),
            "spq_times": (i32, [vp, pd]),
            "spq_level_times": (i32, [vp, pf]),
            "spq_level_flops": (i32, [vp, pd]),
            "spq_factor_flops": (f64, [vp]),
            "spq_rrqr_bytes": (f64, [vp]),
            "spq_pool_bytes": (f64, [vp]),
            "spq_last_error": (C.c_char_p, [vp]),
            "spq_kernel_launches": (C.c_longlong, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _pi(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _pf(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _pd(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def as_csc(A):
    """Accept a scipy sparse matrix or a (colptr, rowidx, values) triple."""
    if isinstance(A, tuple):
        colptr, rowidx, vals = A
        n = len(colptr) - 1
        return (np.ascontiguousarray(colptr, np.int32), np.ascontiguousarray(rowidx, np.int32),
                np.ascontiguousarray(vals, np.float64), n, n)
    import scipy.sparse as sp

    A = sp.csc_matrix(A)
    A.sort_indices()
    return (A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64), A.shape[0], A.shape[1])


def scale_columns(colptr, vals):
    """The driver's column scaling (pspaQR.cpp:133-146), computed by the library."""
    colptr = np.ascontiguousarray(colptr, np.int32)
    out = np.array(vals, dtype=np.float64, copy=True)
    rc = lib().spq_scale_columns(len(colptr) - 1, _pi(colptr), _pd(out))
    if rc:
        raise SpqError("scale_columns", rc, "bad arguments")
    return out


def random_reference(n: int, seed: int) -> np.ndarray:
    """util.cpp:992-1001 ``random(size, seed)``: mt19937, U(-1, 1)."""
    out = np.empty(n)
    lib().spq_random_reference(n, seed, _pd(out))
    return out


def kernel_launches() -> int:
    """Kernels launched by libspaqr_b200.so in this process so far."""
    return int(lib().spq_kernel_launches())


INFO_FIELDS = ("lvl", "merge_lvl", "size", "rank", "parent", "cstart", "sep", "l_lvl", "l_sep", "r_lvl", "r_sep",
               "section", "size_org", "sparsify", "nchildren", "interior")


class ParTree:
    """GPU ParTree: same construction, setters and call order as the reference."""

    def __init__(self, nlevels: int, skip: int = 0):
        h = C.c_void_p()
        rc = lib().spq_create(nlevels, skip, C.byref(h))
        if rc:
            raise SpqError("ParTree", rc, "nlevels must be >= 2 and skip >= 0")
        self._h = h
        self.nlevels = nlevels
        self._A = None

    def close(self):
        if getattr(self, "_h", None):
            lib().spq_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _chk(self, rc: int, what: str):
        if rc != 0:
            raise SpqError(what, rc, (lib().spq_last_error(self._h) or b"").decode())

    # -- setters (tree.cpp:14-21, ptree.cpp:21-23)
    def set_tol(self, tol: float):
        self._chk(lib().spq_set_tol(self._h, tol), "set_tol")

    def set_skip(self, s: int):
        self._chk(lib().spq_set_skip(self._h, s), "set_skip")

    def set_scale(self, s: int):
        self._chk(lib().spq_set_scale(self._h, s), "set_scale")

    def set_order(self, o: float):
        self._chk(lib().spq_set_order(self._h, o), "set_order")

    def set_hsl(self, h: int):
        self._chk(lib().spq_set_hsl(self._h, h), "set_hsl")

    def set_nthreads(self, n: int):
        self._chk(lib().spq_set_nthreads(self._h, n), "set_nthreads")

    def set_verbose(self, v: int):
        self._chk(lib().spq_set_verbose(self._h, v), "set_verbose")

    def set_ttor_log(self, l: int):
        self._chk(lib().spq_set_ttor_log(self._h, l), "set_ttor_log")

    def set_square(self, s: int):
        self._chk(lib().spq_set_square(self._h, s), "set_square")

    def set_pivot_rtol(self, r: float):
        self._chk(lib().spq_set_pivot_rtol(self._h, r), "set_pivot_rtol")

    def set_rrqr_work(self, elems: float, fill: float = 2.0):
        """Cluster sizing of the pivoted QR: elements of the compression matrix
        per CTA and pivot step, and CTAs per SM a level's work is spread over."""
        self._chk(lib().spq_set_rrqr_work(self._h, elems, fill), "set_rrqr_work")

    def set_precision(self, bits: int):
        """32: float factors and preconditioner apply (FP64 SpMV, Krylov loop and
        pivoted QR); 64: plain FP64.  Takes effect at the next assemble."""
        self._chk(lib().spq_set_precision(self._h, bits), "set_precision")

    def set_tensor_cores(self, mode):
        """Float factors' block-reflector applies: 0 / False = CUDA cores, 1 / True =
        3xTF32 tcgen05 MMAs, 2 = tuned per level from the first two factorizations (the
        tensor cores where at least 5 % faster)."""
        self._chk(lib().spq_set_tensor_cores(self._h, int(mode)), "set_tensor_cores")

    def tune_table(self) -> np.ndarray:
        """(nlevels, 3, 3): for updates / left applies / right applies: tensor-core ms,
        CUDA-core ms, choice (1 tensor, 0 CUDA, -1 not tuned yet)."""
        out = np.zeros(9 * self.nlevels, np.float32)
        lib().spq_tune_table(self._h, _pf(out))
        return out.reshape(self.nlevels, 3, 3)

    def set_spin_limit(self, cycles: int):
        """Cycle budget of the preconditioner apply's bounded waits (next factorize)."""
        self._chk(lib().spq_set_spin_limit(self._h, int(cycles)), "set_spin_limit")

    def set_plan_cache(self, on: bool):
        """Reuse a level's descriptor lists when a later factorize meets the same sizes."""
        self._chk(lib().spq_set_plan_cache(self._h, int(bool(on))), "set_plan_cache")

    def plan_hits(self) -> int:
        """Levels whose descriptor lists were reused so far."""
        return int(lib().spq_plan_hits(self._h))

    def set_checks(self, on: bool):
        """Host-side bounds checks of the factorization's descriptors before upload."""
        self._chk(lib().spq_set_checks(self._h, int(bool(on))), "set_checks")

    def debug_corrupt_descriptor(self):
        """Fault injection (tests): the next factorize corrupts one descriptor on the host."""
        self._chk(lib().spq_debug_corrupt_descriptor(self._h), "debug_corrupt_descriptor")

    def set_krylov(self, method: int):
        """0: left GMRES (reference); 1: flexible right-preconditioned GMRES;
        -1: flexible exactly with float factors (default)."""
        self._chk(lib().spq_set_krylov(self._h, method), "set_krylov")

    def set_rank_model(self, model: Optional[dict], oversample: int = 32):
        """Learned ranks from ``model`` (``params``, ``mean``, ``std`` float32
        arrays, e.g. :func:`load_rank_model`); ``None`` restores the plain
        pivoted QR of every interface."""
        if model is None:
            self._chk(lib().spq_set_rank_model(self._h, None, None, None, 0), "set_rank_model")
            return
        self._model = {k: np.ascontiguousarray(model[k], dtype=np.float32) for k in ("params", "mean", "std")}
        m = self._model
        self._chk(lib().spq_set_rank_model(self._h, _pf(m["params"]), _pf(m["mean"]), _pf(m["std"]), oversample),
                  "set_rank_model")
        self._chk(lib().spq_set_rank_margin(self._h, float(model.get("margin", 0.0))), "set_rank_margin")

    def set_sketch_tuning(self, sketch_tol: float = 0.1, smem: bool = False):
        """Stop of the sketch's pivoted QR (x tol) and its shared-memory mode."""
        self._chk(lib().spq_set_sketch_tuning(self._h, sketch_tol, int(smem)), "set_sketch_tuning")

    def learned_counts(self) -> dict:
        out = (C.c_longlong * 3)()
        self._chk(lib().spq_learned_counts(self._h, out), "learned_counts")
        return {"accepted": out[0], "fallback": out[1], "sketch_columns": out[2]}

    def set_rank_log(self, on: bool = True):
        self._chk(lib().spq_set_rank_log(self._h, int(on)), "set_rank_log")

    def rank_log(self) -> dict:
        """Logged (features, kept rank, min(m, w), level) of the sparsified interfaces."""
        n = lib().spq_rank_log_count(self._h)
        _, nf = rank_model_size()
        out = {"features": np.zeros((n, nf), np.float32), "rank": np.zeros(n, np.int32),
               "kmin": np.zeros(n, np.int32), "level": np.zeros(n, np.int32)}
        if n:
            self._chk(lib().spq_rank_log(self._h, _pf(out["features"]), _pi(out["rank"]), _pi(out["kmin"]),
                                         _pi(out["level"])), "rank_log")
        return out

    def clear_rank_log(self):
        self._chk(lib().spq_rank_log_clear(self._h), "rank_log_clear")

    def set_Xcoo(self, X: np.ndarray):
        """Coordinates as a dim x n array (tree.cpp:21)."""
        X = np.asfortranarray(X, dtype=np.float64)
        self._chk(lib().spq_set_coords(self._h, X.shape[0], X.shape[1], _pd(X)), "set_Xcoo")

    def set_coords_tensor(self, n: int, d: int):
        """linspace_nd(n, d) coordinates (util.cpp:901-930)."""
        self._chk(lib().spq_set_coords_tensor(self._h, n, d), "set_coords_tensor")

    def set_stream(self, stream_ptr: int):
        self._chk(lib().spq_set_stream(self._h, C.c_void_p(stream_ptr)), "set_stream")

    # -- pipeline
    def partition(self, A):
        colptr, rowidx, vals, nr, nc = as_csc(A)
        self._A = (colptr, rowidx, vals)
        self._chk(lib().spq_partition(self._h, nr, nc, _pi(colptr), _pi(rowidx), _pd(vals)), "partition")

    def assemble(self, A=None):
        self._chk(lib().spq_assemble(self._h), "assemble")

    def factorize(self) -> int:
        self._chk(lib().spq_factorize(self._h), "factorize")
        return 0

    def solve(self, b: np.ndarray, x: Optional[np.ndarray] = None) -> np.ndarray:
        """One-shot solve with a global right-hand side (ptree.cpp:2268-2785)."""
        b = np.ascontiguousarray(b, np.float64)
        out = np.zeros_like(b) if x is None else x
        self._chk(lib().spq_solve_global(self._h, _pd(b), _pd(out)), "solve")
        return out

    def solve_inplace(self, x: np.ndarray) -> np.ndarray:
        """Preconditioner apply on a permuted local vector (ptree.cpp:2788-3210)."""
        if x.dtype != np.float64 or not x.flags.c_contiguous:
            raise TypeError("x must be a contiguous float64 array")
        self._chk(lib().spq_solve_inplace(self._h, _pd(x)), "solve")
        return x

    def solve_inplace_device(self, ptr: int):
        self._chk(lib().spq_solve_inplace_device(self._h, C.c_void_p(ptr)), "solve")

    def spmv(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty_like(x)
        self._chk(lib().spq_spmv(self._h, _pd(x), _pd(y)), "spmv")
        return y

    def backward_error(self, nprobe: int = 3, probes: Optional[np.ndarray] = None, seed: int = 2021) -> np.ndarray:
        """||A z - u|| / ||u||, z = M^{-1} u, for nprobe probe vectors u (permuted
        order): the factorization's relative backward error ||(A P - Q R) z|| / ||Q R z||.
        ``probes`` (n x nprobe) gives them; otherwise u ~ N(0,1) from mt19937_64(seed + p)."""
        eta = np.zeros(nprobe)
        U = None
        if probes is not None:
            U = np.asfortranarray(probes, dtype=np.float64).reshape(self.nrows_local(), nprobe, order="F")
        self._chk(lib().spq_factor_backward_error(self._h, nprobe, _pd(U) if U is not None else None, seed, _pd(eta)),
                  "backward_error")
        return eta

    def nrows_local(self) -> int:
        return lib().spq_n(self._h)

    def ncols_local(self) -> int:
        return lib().spq_n(self._h)

    def distribute_x(self, x: np.ndarray, x_dist: np.ndarray):
        x = np.ascontiguousarray(x, np.float64)
        self._chk(lib().spq_distribute_x(self._h, _pd(x), _pd(x_dist)), "distribute_x")

    def extract_x(self, x_local: np.ndarray) -> np.ndarray:
        x_local = np.ascontiguousarray(x_local, np.float64)
        out = np.empty_like(x_local)
        self._chk(lib().spq_extract_x(self._h, _pd(x_local), _pd(out)), "extract_x")
        return out

    # -- introspection
    def perm(self) -> np.ndarray:
        p = np.empty(self.nrows_local(), np.int32)
        self._chk(lib().spq_get_perm(self._h, _pi(p)), "perm")
        return p

    def num_clusters(self) -> int:
        return lib().spq_num_clusters(self._h)

    def level_range(self, lvl: int):
        f, c = C.c_int(), C.c_int()
        self._chk(lib().spq_level_range(self._h, lvl, C.byref(f), C.byref(c)), "level_range")
        return f.value, c.value

    def cluster(self, order: int) -> dict:
        info = np.zeros(16, np.int32)
        self._chk(lib().spq_cluster_info(self._h, order, _pi(info)), "cluster_info")
        return dict(zip(INFO_FIELDS, info.tolist()))

    def clusters(self):
        return [self.cluster(o) for o in range(self.num_clusters())]

    def num_edges(self) -> int:
        return lib().spq_num_edges(self._h)

    def find_edge(self, n1: int, n2: int) -> int:
        return lib().spq_find_edge(self._h, n1, n2)

    def block(self, n1: int, n2: int):
        shape = np.zeros(3, np.int32)
        if lib().spq_get_block(self._h, n1, n2, None, _pi(shape)) != 0:
            return None
        r, c, ld = (int(v) for v in shape)
        buf = np.zeros(max(ld * c, 1))
        lib().spq_get_block(self._h, n1, n2, _pd(buf), _pi(shape))
        return buf[: ld * c].reshape(c, ld).T[:r, :]

    def factor(self, order: int, which: int):
        """0: diagonal-QR T, 1: scaling T, 2: sparsification V, 3: its T (None if absent)."""
        shape = np.zeros(3, np.int32)
        if lib().spq_get_factor(self._h, order, which, None, _pi(shape)) != 0:
            return None
        r, c = int(shape[0]), int(shape[1])
        buf = np.zeros(max(r * c, 1))
        lib().spq_get_factor(self._h, order, which, _pd(buf), _pi(shape))
        return buf[: r * c].reshape(c, r).T

    def times(self) -> dict:
        t = np.zeros(5)
        lib().spq_times(self._h, _pd(t))
        return dict(zip(("partition", "assemble", "factorize", "solve", "gmres"), t.tolist()))

    LEVEL_PHASES = ("chains", "updates", "scale_qr", "scale_apply", "rrqr", "compress_apply", "merge", "total")

    def level_times(self) -> np.ndarray:
        """(nlevels, 8) milliseconds per phase, columns as LEVEL_PHASES."""
        out = np.zeros(8 * self.nlevels, np.float32)
        lib().spq_level_times(self._h, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out.reshape(self.nlevels, 8)

    def level_flops(self) -> np.ndarray:
        """(nlevels, 6) nominal flops per phase, columns as LEVEL_PHASES[:6]."""
        out = np.zeros(6 * self.nlevels, np.float64)
        lib().spq_level_flops(self._h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out.reshape(self.nlevels, 6)

    def factor_flops(self) -> float:
        return lib().spq_factor_flops(self._h)

    def rrqr_bytes(self) -> float:
        """Compression-matrix bytes the pivoted QR read in the last factorize."""
        return lib().spq_rrqr_bytes(self._h)

    def pool_bytes(self) -> float:
        return lib().spq_pool_bytes(self._h)


def block_gmres(M: ParTree, B: np.ndarray, iters: int = 100, tol: float = 1e-10):
    """Flexible GMRES of the columns of B (n x nrhs, permuted local order) in
    lockstep, one block preconditioner apply per iteration; B is overwritten by
    the solutions.  Returns (iterations, true relative residuals) per column."""
    if B.dtype != np.float64 or not B.flags.f_contiguous or B.ndim != 2:
        raise TypeError("B must be a Fortran-ordered float64 n x nrhs array")
    n, nrhs = B.shape
    k = np.zeros(nrhs, np.int32)
    rr = np.zeros(nrhs)
    M._chk(lib().spq_gmres_block(M._h, _pd(B), nrhs, n, iters, tol, _pi(k), _pd(rr)), "gmres_block")
    return k, rr


def dist_gmres(A, b: np.ndarray, M: ParTree, iters: int = 300, tol: float = 1e-12, verb: bool = True,
               hist: Optional[list] = None):
    """is.cpp:447-527: b (permuted local order) is overwritten by the solution.

    Returns ``(k, relres)``: the reference's iteration index at the break and the
    true relative residual ||b0 - A x|| / ||b0|| (pspaQR.cpp:264-268).
    """
    if b.dtype != np.float64 or not b.flags.c_contiguous:
        raise TypeError("b must be a contiguous float64 array")
    k = C.c_int()
    rr = C.c_double()
    h = np.zeros(iters)
    M._chk(lib().spq_gmres(M._h, _pd(b), iters, tol, C.byref(k), C.byref(rr), _pd(h), iters), "gmres")
    if hist is not None:
        hist.extend(h[: k.value + 1].tolist())
    return k.value, rr.value


# ---------------------------------------------------------------- rank MLP
def rank_model_size():
    """(number of MLP parameters, number of interface features)."""
    a, b = C.c_int(), C.c_int()
    lib().spq_rank_model_size(C.byref(a), C.byref(b))
    return a.value, b.value


def _mlp_check(rc, what):
    if rc != 0:
        raise SpqError(what, rc, (lib().spq_mlp_last_error() or b"").decode())


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


def mlp_loss_grad(params, X, y):
    """Loss mean((sigmoid(z) - y)^2) and its gradient, on the GPU."""
    P, F = rank_model_size()
    params, X, y = _f32(params, (P,)), _f32(X), _f32(y)
    loss, grad = np.zeros(1, np.float32), np.zeros(P, np.float32)
    _mlp_check(lib().spq_mlp_loss_grad(_pf(params), _pf(X), _pf(y), len(y), _pf(loss), _pf(grad)), "mlp_loss_grad")
    return float(loss[0]), grad


def mlp_predict(params, X):
    P, F = rank_model_size()
    params, X = _f32(params, (P,)), _f32(X)
    out = np.zeros(len(X), np.float32)
    _mlp_check(lib().spq_mlp_predict(_pf(params), _pf(X), len(X), _pf(out)), "mlp_predict")
    return out


def mlp_train(params, X, y, epochs: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0):
    """Adam training on the GPU; returns (params, per-epoch loss)."""
    P, F = rank_model_size()
    params = _f32(params, (P,)).copy()
    X, y = _f32(X), _f32(y)
    hist = np.zeros(max(epochs, 1), np.float32)
    _mlp_check(lib().spq_mlp_train(_pf(params), _pf(X), _pf(y), len(y), epochs, batch, lr, seed, _pf(hist)),
               "mlp_train")
    return params, hist[:epochs]


def mlp_init(seed: int = 0):
    """He-initialised parameters in the library's layout."""
    P, F = rank_model_size()
    H = 64
    rng = np.random.default_rng(seed)
    W1 = rng.normal(0, np.sqrt(2.0 / F), (H, F))
    W2 = rng.normal(0, np.sqrt(2.0 / H), (H, H))
    w3 = rng.normal(0, np.sqrt(1.0 / H), H)
    p = np.concatenate([W1.ravel(), np.zeros(H), W2.ravel(), np.zeros(H), w3, [0.0]]).astype(np.float32)
    assert p.size == P
    return p


def load_rank_model(path: Optional[str] = None, tol: Optional[float] = None) -> dict:
    """The trained rank model shipped with the package (rank_model/rank_mlp.npz).
    With ``tol``, the sketch margin calibrated for the nearest training tolerance
    (``margin``: an upper quantile of the network's error on its training pairs)
    comes with it; without, the margin is 0."""
    path = path or os.path.join(_HERE, "rank_model", "rank_mlp.npz")
    z = np.load(path)
    out = {k: z[k].astype(np.float32) for k in ("params", "mean", "std")}
    meta = json.loads(str(z["meta"])) if "meta" in z.files else {}
    if tol is not None and meta.get("margin_by_tol"):
        tols = [float(k) for k in meta["margin_by_tol"]]
        near = min(tols, key=lambda x: abs(np.log10(x) - np.log10(tol)))
        out["margin"] = float(meta["margin_by_tol"][repr(near) if repr(near) in meta["margin_by_tol"] else str(near)])
    return out
