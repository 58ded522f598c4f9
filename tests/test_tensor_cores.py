"""Tensor-core (tcgen05, 3xTF32) left applies of the float factorization against
the same factorization on the CUDA cores and against the FP64 oracle.

Both float variants compute the same products in a different order and with a
different rounding of the operands (3xTF32 keeps about 21 bits of each product),
so their factors agree to float rounding amplified by the elimination:
1e-4 relative on the top separator's R and on the preconditioner apply.  The
ranks come from the FP64 pivoted QR of the float blocks and agree on almost every
interface.  Against the FP64 oracle the float factor's backward error matches the
oracle's to 20 % (the sparsification tolerance dominates the float rounding), and
flexible GMRES reaches the 1e-10 residual."""
import numpy as np
import pytest

from oracle.oracle import OracleTree, random_reference
from pspaqr_public_b200 import ParTree, dist_gmres, scale_columns
from pspaqr_public_b200 import matrices as M

pytestmark = pytest.mark.gpu


def _float_tree(cp, ri, v, n, L, tol, tc):
    t = ParTree(L, 0)
    t.set_tol(tol)
    t.set_coords_tensor(n, 3)
    t.set_precision(32)
    t.set_tensor_cores(tc)
    t.partition((cp, ri, scale_columns(cp, v)))
    t.assemble()
    t.factorize()
    return t


def _relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("n,L", [(8, 3), (16, 6), (32, 8)])
def test_tensor_cores_match_cuda_cores(n, L):
    cp, ri, v = M.diffusion_lognormal(n, 3, seed=2)
    a = _float_tree(cp, ri, v, n, L, 1e-2, True)
    b = _float_tree(cp, ri, v, n, L, 1e-2, False)
    ra = np.array([c["rank"] for c in a.clusters()])
    rb = np.array([c["rank"] for c in b.clusters()])
    assert np.mean(ra == rb) >= 0.98, np.mean(ra == rb)
    x = random_reference(n ** 3, 3)
    xa = a.solve_inplace(x.copy())
    xb = b.solve_inplace(x.copy())
    # block by block only while the two float factorizations take the same
    # pivots: from 32^3 on, rounding flips near-tied pivots of the pivoted QR and
    # the bases differ while the ranks agree; the backward error judges them
    if np.array_equal(ra, rb) and n <= 16:
        top = a.level_range(L - 1)[0]
        Ra, Rb = np.triu(a.block(top, top)), np.triu(b.block(top, top))
        assert np.abs(Ra - Rb).max() <= 1e-4 * np.abs(Rb).max()
        assert _relerr(xa, xb) <= 1e-4
    ea, eb = a.backward_error(2), b.backward_error(2)
    assert np.all(ea <= 1.1 * eb + 1e-6), (ea, eb)


def test_tensor_cores_against_fp64_oracle():
    n, L, tol = 32, 8, 1e-2
    cp, ri, v = M.diffusion_lognormal(n, 3, seed=2)
    t = _float_tree(cp, ri, v, n, L, tol, True)
    o = OracleTree(L, 0, tol, 4)
    o.set_matrix(cp, ri, v)
    o.set_coords_tensor(n, 3)
    o.partition()
    o.assemble()
    o.factorize()
    N = n ** 3
    U = np.stack([np.random.default_rng(50 + p).standard_normal(N) for p in range(2)], axis=1)
    eta_o = np.array([np.linalg.norm(o.spmv(o.solve_inplace(U[:, p])) - U[:, p]) / np.linalg.norm(U[:, p])
                      for p in range(2)])
    eta_t = t.backward_error(2, U)
    assert np.all(np.abs(eta_t / eta_o - 1) < 0.2), (eta_t, eta_o)
    x = M.rhs_normal(N, 2)
    k, rr = dist_gmres(None, x, t, 300, 1e-10)
    assert rr <= 1e-10
