"""Several right-hand sides solved together (BASELINE config 5 at a reduced size:
2D upwinded convection-diffusion, 128^2, 8 levels, tol 1e-2).

* The block preconditioner apply (nrhs concurrent sweeps in one graph) equals the
  single-vector apply column by column, bit for bit: the same kernels on separate
  workspaces.
* Lockstep flexible GMRES gives every column the iteration count and solution of
  the single-right-hand-side flexible GMRES, and a true residual <= 1e-10.
* Against the FP64 oracle (left-preconditioned GMRES of each column, the
  reference method): the solutions agree to the accuracy the residual allows.
* With float factors (tensor-core updates) every column still reaches 1e-10.
"""
import numpy as np
import pytest

from oracle.oracle import OracleTree
from pspaqr_public_b200 import ParTree, dist_gmres, scale_columns
from pspaqr_public_b200 import matrices as M
from pspaqr_public_b200.tree import block_gmres, lib

pytestmark = pytest.mark.gpu
N, L, TOL, NRHS = 128, 8, 1e-2, 4


def _tree(precision=64):
    cp, ri, v = M.convection_diffusion_2d(N)
    t = ParTree(L, 0)
    t.set_tol(TOL)
    t.set_coords_tensor(N, 2)
    t.set_precision(precision)
    t.partition((cp, ri, scale_columns(cp, v)))
    t.assemble()
    t.factorize()
    return t


def test_block_apply_equals_single_applies():
    import ctypes as C

    import torch

    t = _tree()
    n = N * N
    B = M.rhs_normal(n, 4, NRHS)
    X = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()  # column r = row r of X (contiguous)
    torch.cuda.synchronize()
    rc = lib().spq_solve_block_device(t._h, C.c_void_p(X.data_ptr()), NRHS, n)
    assert rc == 0, lib().spq_last_error(t._h)
    torch.cuda.synchronize()  # the library runs on its own stream
    Xb = X.cpu().numpy()
    for r in range(NRHS):
        x = t.solve_inplace(np.ascontiguousarray(B[:, r]))
        assert np.array_equal(Xb[r], x)


@pytest.mark.parametrize("precision", [64, 32])
def test_lockstep_fgmres_matches_single_solves(precision):
    t = _tree(precision)
    n = N * N
    B = M.rhs_normal(n, 4, NRHS)
    X = np.asfortranarray(B.copy())
    k, rr = block_gmres(t, X, 100, 1e-10)
    assert np.all(rr <= 1e-10), rr
    t.set_krylov(1)
    for r in range(NRHS):
        x = np.ascontiguousarray(B[:, r])
        kr, rrr = dist_gmres(None, x, t, 100, 1e-10)
        assert kr == k[r]
        assert np.linalg.norm(X[:, r] - x) <= 1e-12 * np.linalg.norm(x)


def test_block_solutions_against_fp64_oracle():
    t = _tree()
    cp, ri, v = M.convection_diffusion_2d(N)
    o = OracleTree(L, 0, TOL, 4)
    o.set_matrix(cp, ri, v)
    o.set_coords_tensor(N, 2)
    o.partition()
    o.assemble()
    o.factorize()
    n = N * N
    B = M.rhs_normal(n, 4, NRHS)
    X = np.asfortranarray(B.copy())
    k, rr = block_gmres(t, X, 100, 1e-10)
    for r in range(NRHS):
        xo, ko, rro, _ = o.gmres(np.ascontiguousarray(B[:, r]), 300, 1e-12)
        assert rro <= 1e-10
        # both residuals <= 1e-10: the solutions differ by at most cond(A) times that
        assert np.linalg.norm(X[:, r] - xo) <= 1e-6 * np.linalg.norm(xo)
        assert abs(int(k[r]) - ko) <= 2
