"""Failure detection through the C ABI: every failure is made on the host (a value,
a descriptor, a cycle budget), none faults or hangs the GPU, and the tree is usable
again after it.

* a non-finite matrix value is rejected by partition (-2), before any GPU work;
* a zero pivot (an exactly zero column) is reported by the factorization's device
  status word (-13) after the level that met it;
* a descriptor moved out of the block pool on the host is caught by the host-side
  bounds check before its upload (-5);
* a zero cycle budget makes the preconditioner apply's bounded waits run out: the
  GMRES call fails with -12, and the next call with the default budget succeeds
  (the status word is cleared on entry).
"""
import numpy as np
import pytest

from pspaqr_public_b200 import ParTree, SpqError, dist_gmres, random_reference, scale_columns
from pspaqr_public_b200 import matrices as M


def _tree(n, d, L, tol=1e-2):
    t = ParTree(L, 0)
    t.set_tol(tol)
    t.set_coords_tensor(n, d)
    return t


def test_non_finite_value_rejected_by_partition():
    cp, ri, v = M.laplacian(8, 2)
    v = scale_columns(cp, v)
    v[7] = np.nan
    t = _tree(8, 2, 3)
    with pytest.raises(SpqError) as e:
        t.partition((cp, ri, v))
    assert e.value.status == -2 and "not finite" in str(e.value)
    v[7] = np.inf
    with pytest.raises(SpqError):
        _tree(8, 2, 3).partition((cp, ri, v))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [64, 32])
def test_zero_pivot_reported_by_the_device_status_word(precision):
    n, d, L = 16, 3, 6
    cp, ri, v = M.laplacian(n, d)
    v = scale_columns(cp, v)
    col = 1234
    v[cp[col]:cp[col + 1]] = 0.0  # an exactly zero column: R(j, j) = 0 in its cluster's QR
    t = _tree(n, d, L)
    t.set_precision(precision)
    t.partition((cp, ri, v))
    t.assemble()
    with pytest.raises(SpqError) as e:
        t.factorize()
    assert e.value.status == -13 and "zero pivot" in str(e.value)
    # the same tree with a regular matrix factorizes and solves
    cp, ri, v = M.laplacian(n, d)
    t.partition((cp, ri, scale_columns(cp, v)))
    t.assemble()
    t.factorize()
    k, rr = dist_gmres(None, random_reference(n ** d, 1), t, 100, 1e-10)
    assert rr < 1e-9


@pytest.mark.gpu
def test_corrupted_descriptor_caught_before_launch():
    n, d, L = 16, 3, 6
    cp, ri, v = M.laplacian(n, d)
    t = _tree(n, d, L)
    t.partition((cp, ri, scale_columns(cp, v)))
    t.assemble()
    t.debug_corrupt_descriptor()
    with pytest.raises(SpqError) as e:
        t.factorize()
    assert e.value.status == -5 and "outside the block pool" in str(e.value)
    # checks stay on; a fresh assembly factorizes cleanly through them
    t.assemble()
    t.factorize()
    k, rr = dist_gmres(None, random_reference(n ** d, 2), t, 100, 1e-10)
    assert rr < 1e-9


@pytest.mark.gpu
def test_bounded_wait_timeout_then_recovery():
    n, d, L = 32, 3, 8
    cp, ri, v = M.laplacian(n, d)
    t = _tree(n, d, L)
    t.partition((cp, ri, scale_columns(cp, v)))
    t.set_spin_limit(0)
    t.assemble()
    t.factorize()
    b = random_reference(n ** d, 3)
    with pytest.raises(SpqError) as e:
        dist_gmres(None, b.copy(), t, 50, 1e-10)
    assert e.value.status == -12
    t.set_spin_limit(2_000_000_000)
    t.assemble()
    t.factorize()
    k, rr = dist_gmres(None, b.copy(), t, 100, 1e-10)
    assert rr < 1e-9
