"""Allocation-free GMRES (spq_gmres_device_noalloc) against spq_gmres_device.

Both entry points are called through the C ABI on the same factorization and
right-hand side; the allocation-free one twice in a row, each result compared
with the cached-workspace one.  Collected last so it also runs after every
other GPU test in the same process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, D, L, MAXIT, TOL = 32, 3, 8, 60, 1e-10


@pytest.fixture(scope="module")
def tree():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from pspaqr_public_b200 import ParTree, scale_columns
    from pspaqr_public_b200 import matrices as M

    cp, ri, v = M.diffusion_lognormal(N, D, seed=2)
    t = ParTree(L, 0)
    t.set_tol(1e-2)
    t.set_coords_tensor(N, D)
    t.partition((cp, ri, scale_columns(cp, v)))
    t.assemble()
    t.factorize()
    return t


def _gmres(t, b, noalloc, maxit=MAXIT):
    import torch
    from pspaqr_public_b200.tree import lib

    x = torch.from_numpy(b.copy()).cuda()
    torch.cuda.synchronize()
    k, rr = C.c_int(), C.c_double()
    if noalloc:
        rc = lib().spq_gmres_device_noalloc(t._h, C.c_void_p(x.data_ptr()), maxit, TOL, C.byref(k), C.byref(rr))
    else:
        rc = lib().spq_gmres_device(t._h, C.c_void_p(x.data_ptr()), maxit, TOL, C.byref(k), C.byref(rr), None, 0)
    msg = (lib().spq_last_error(t._h) or b"").decode()
    return rc, msg, x.cpu().numpy(), k.value, rr.value


def test_noalloc_matches_cached_workspace(tree):
    from pspaqr_public_b200 import random_reference

    b = random_reference(N**D, 11)
    rc, msg, x_ref, k_ref, rr_ref = _gmres(tree, b, noalloc=False)
    assert rc == 0, msg
    assert rr_ref < 1e-9
    for _ in range(2):
        rc, msg, x, k, rr = _gmres(tree, b, noalloc=True)
        assert rc == 0, msg
        assert k == k_ref
        assert np.linalg.norm(x - x_ref) <= 1e-12 * np.linalg.norm(x_ref)
        assert abs(rr - rr_ref) <= 1e-12 + 1e-6 * rr_ref


def test_noalloc_rejects_oversized_requests(tree):
    from pspaqr_public_b200 import random_reference

    b = random_reference(N**D, 12)
    rc, msg, _, _, _ = _gmres(tree, b, noalloc=True, maxit=101)
    assert rc != 0 and "maxit" in msg


def test_noalloc_later_calls_commit_no_device_memory(tree):
    """The first call loads the library module that holds the fixed array (48 MiB);
    a later call must leave the device's free memory unchanged."""
    import torch
    from pspaqr_public_b200 import random_reference

    b = random_reference(N**D, 13)
    x = torch.from_numpy(b.copy()).cuda()
    rc, msg, _, _, _ = _gmres(tree, b, noalloc=True)
    assert rc == 0, msg
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc, msg, _, _, _ = _gmres(tree, b, noalloc=True)
    assert rc == 0, msg
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    del x
    assert free1 == free0


def test_noalloc_rejects_a_basis_larger_than_the_array():
    """48^3 unknowns with maxit 100 need 110,592 * 103 + 1128 doubles and more:
    beyond the fixed 6,291,456 the call fails with the size it needed."""
    from pspaqr_public_b200 import ParTree, random_reference, scale_columns
    from pspaqr_public_b200 import matrices as M

    n = 48
    cp, ri, v = M.laplacian(n, 3)
    t = ParTree(8, 0)
    t.set_tol(1e-1)
    t.set_coords_tensor(n, 3)
    t.partition((cp, ri, scale_columns(cp, v)))
    t.assemble()
    t.factorize()
    assert n**3 * (100 + 3) > 6_291_456
    rc, msg, _, _, _ = _gmres(t, random_reference(n**3, 14), noalloc=True, maxit=100)
    assert rc == -14 and "doubles" in msg, (rc, msg)
    # within the bound the same tree solves
    rc, msg, _, _, rr = _gmres(t, random_reference(n**3, 14), noalloc=True, maxit=40)
    assert rc == 0, msg
