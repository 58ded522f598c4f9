"""Generate the golden fixtures of the CPU oracle (tests/golden/*.npz).

The reference itself cannot be built or run here (Eigen, MPI, TaskTorrent and
the LAPACKE headers are absent), so these fixtures freeze the oracle's outputs
on the small configurations: the nested-dissection permutation, per-cluster
kept ranks, the diagonal of the top R block, the one-shot preconditioner
residual and the GMRES iteration count / history.  Regenerate with
``python tests/golden/make_golden.py``.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import OracleTree, random_reference  # noqa: E402
from pspaqr_public_b200 import matrices as M  # noqa: E402

CASES = {
    # name: (grid n, dim, nlevels, tol, skip, gmres tol)
    "lapl2d_16_l3": (16, 2, 3, 1e-2, 0, 1e-12),
    "lapl2d_64_l6": (64, 2, 6, 1e-2, 0, 1e-12),
    "lapl2d_64_l6_skip1": (64, 2, 6, 1e-2, 1, 1e-12),
    "lapl3d_16_l6": (16, 3, 6, 1e-2, 0, 1e-12),
}


def run_case(n, d, L, tol, skip, gtol):
    cp, ri, v = M.laplacian(n, d)
    o = OracleTree(L, skip, tol, 1)
    o.set_matrix(cp, ri, v)
    o.set_coords_tensor(n, d)
    o.partition()
    o.assemble()
    o.factorize()
    N = n ** d
    cls = o.clusters()
    top = o.level(L - 1)[0][0]
    R = o.block(top, top)
    b = random_reference(N, 2021)
    x = o.solve_inplace(b)
    res = np.linalg.norm(b - o.spmv(x)) / np.linalg.norm(b)
    xg, k, rr, hist = o.gmres(b.copy(), 300, gtol)
    bn = M.rhs_normal(N, 0)
    xg2, k2, rr2, hist2 = o.gmres(bn.copy(), 300, gtol)
    return dict(
        perm=o.perm(),
        rank=np.array([c["rank"] for c in cls], np.int32),
        size_org=np.array([c["cols_org"] for c in cls], np.int32),
        sparsified=np.array([c["sparsified"] for c in cls], np.int32),
        top_rdiag=np.abs(np.diag(R)),
        precond_residual=np.array(res),
        precond_x=x,
        gmres_iters=np.array(k),
        gmres_relres=np.array(rr),
        gmres_hist=hist,
        gmres_iters_normal=np.array(k2),
        gmres_relres_normal=np.array(rr2),
    )


def main():
    for name, case in CASES.items():
        out = run_case(*case)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "ranks kept", int(out["rank"].sum()), "gmres", int(out["gmres_iters"]), float(out["gmres_relres"]))


if __name__ == "__main__":
    main()
