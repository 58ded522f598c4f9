"""Generate the 64^3 golden fixtures of the CPU oracle (tests/golden/*_64_*.npz).

These freeze the oracle's outputs at the size the headline workload runs:

* ``lapl3d_64_t1e-2``: 3D 7-point Laplacian on 64^3, 12 levels, tol 1e-2;
* ``diff3d_64_t1e-2`` / ``diff3d_64_t1e-3``: the variable-coefficient diffusion
  matrix -div(k grad u), k = exp(g), g a Gaussian random field (correlation
  length 8, variance 1, seed 2), 12 levels, tol 1e-2 and 1e-3.

A full 262,144-entry vector would make the fixtures large, so vectors are kept
as size-independent summaries: 4096 entries at seeded positions, the 2-norm, and
8 projections g_k^T x / sqrt(N) on seeded Gaussian vectors (``summary``).  The
permutation is kept as its SHA-256 digest.  Per-cluster kept ranks, the
diagonal of the top separator's R, the GMRES iteration counts and the factor
backward error estimate (``backward_error``) are stored in full.

Regenerate with ``python tests/golden/make_golden_64.py`` (a few minutes on 8
host cores; OpenMP threads = all cores).
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import OracleTree, random_reference  # noqa: E402
from pspaqr_public_b200 import matrices as M  # noqa: E402

N_SAMPLES = 4096
N_PROJ = 8
N_PROBES = 3

CASES = {
    # name: (matrix builder, grid n, dim, nlevels, tol, N(0,1) rhs seed)
    "lapl3d_64_t1e-2": (lambda: M.laplacian(64, 3), 64, 3, 12, 1e-2, 1),
    "diff3d_64_t1e-2": (lambda: M.diffusion_lognormal(64, 3, seed=2), 64, 3, 12, 1e-2, 2),
    "diff3d_64_t1e-3": (lambda: M.diffusion_lognormal(64, 3, seed=2), 64, 3, 12, 1e-3, 2),
}


def sample_index(n: int) -> np.ndarray:
    return np.sort(np.random.default_rng(777).choice(n, N_SAMPLES, replace=False))


def projections(n: int) -> np.ndarray:
    return np.random.default_rng(778).standard_normal((N_PROJ, n)) / np.sqrt(n)


def summary(x: np.ndarray, idx: np.ndarray, P: np.ndarray) -> dict:
    return dict(samples=x[idx], norm=np.array(np.linalg.norm(x)), proj=P @ x)


def probe_rhs(n: int, p: int) -> np.ndarray:
    """Right-hand side of backward-error probe p: N(0,1) from seed 9000 + p."""
    return np.random.default_rng(9000 + p).standard_normal(n)


def backward_error(solve, spmv, n: int) -> np.ndarray:
    """||A z - u|| / ||u|| with z = M^{-1} u for the probe vectors u: the factor's
    relative backward error ||(A P - Q R) z|| / ||Q R z|| in those directions."""
    out = []
    for p in range(N_PROBES):
        u = probe_rhs(n, p)
        z = solve(u.copy())
        out.append(np.linalg.norm(spmv(z) - u) / np.linalg.norm(u))
    return np.array(out)


def run_case(build, n, d, L, tol, seed, threads):
    cp, ri, v = build()
    o = OracleTree(L, 0, tol, threads)
    o.set_matrix(cp, ri, v)
    o.set_coords_tensor(n, d)
    t0 = time.time()
    o.partition()
    o.assemble()
    o.factorize()
    tf = time.time() - t0
    N = n ** d
    idx, P = sample_index(N), projections(N)
    cls = o.clusters()
    top = o.level(L - 1)[0][0]
    R = o.block(top, top)
    b = random_reference(N, 2021)
    x = o.solve_inplace(b)
    _, k, rr, hist = o.gmres(b.copy(), 300, 1e-10)
    bn = M.rhs_normal(N, seed)
    xn, kn, rrn, _ = o.gmres(bn.copy(), 300, 1e-10)
    out = dict(
        perm_sha256=np.array(hashlib.sha256(o.perm().astype(np.int32).tobytes()).hexdigest()),
        rank=np.array([c["rank"] for c in cls], np.int32),
        size_org=np.array([c["cols_org"] for c in cls], np.int32),
        sparsified=np.array([c["sparsified"] for c in cls], np.int8),
        top_rdiag=np.abs(np.diag(R)),
        gmres_iters=np.array(k),
        gmres_relres=np.array(rr),
        gmres_hist=hist,
        gmres_iters_normal=np.array(kn),
        gmres_relres_normal=np.array(rrn),
        backward_error=backward_error(o.solve_inplace, o.spmv, N),
    )
    for key, val in summary(x, idx, P).items():
        out["precond_x_" + key] = val
    for key, val in summary(xn, idx, P).items():
        out["gmres_x_normal_" + key] = val
    return out, tf


def main(names=None):
    threads = os.cpu_count() or 1
    for name, case in CASES.items():
        if names and name not in names:
            continue
        out, tf = run_case(*case, threads)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(f"{name}: factorize {tf:.1f} s, ranks kept {int(out['rank'].sum())}, top {out['top_rdiag'].size}, "
              f"gmres {int(out['gmres_iters'])} / {int(out['gmres_iters_normal'])}, "
              f"backward error {out['backward_error'].max():.3e}", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
