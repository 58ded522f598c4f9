"""GPU path (C ABI) against the CPU oracle: ordering, kept ranks, factors, the
preconditioner apply and GMRES.  Tolerances: FP64 factors and the solve agree to
1e-10 relative (the kernels and LAPACK differ only in summation order); integer
outputs (ranks, permutation, iteration counts) are exact."""
import os

import numpy as np
import pytest

from oracle.oracle import OracleTree, random_reference
from pspaqr_public_b200 import ParTree, dist_gmres, scale_columns
from pspaqr_public_b200 import matrices as M

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
RTOL = 1e-10


def _matrix(kind, n, d):
    if kind == "lapl":
        return M.laplacian(n, d)
    if kind == "diff":
        return M.diffusion_lognormal(n, d, seed=2)
    if kind == "chan":
        return M.diffusion_binary(n, d, seed=3)
    return M.convection_diffusion_2d(n)


def _pair(kind, n, d, L, tol, skip=0):
    cp, ri, v = _matrix(kind, n, d)
    t = ParTree(L, skip)
    t.set_tol(tol)
    t.set_coords_tensor(n, d)
    t.partition((cp, ri, scale_columns(cp, v)))
    t.assemble()
    t.factorize()
    o = OracleTree(L, skip, tol, 4)
    o.set_matrix(cp, ri, v)
    o.set_coords_tensor(n, d)
    o.partition()
    o.assemble()
    o.factorize()
    return t, o


def _relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("kind,n,d,L", [("lapl", 16, 2, 4), ("lapl", 8, 3, 4), ("convdiff", 16, 2, 3)])
def test_exact_without_sparsification(kind, n, d, L):
    t, o = _pair(kind, n, d, L, 0.0)
    N = n ** d
    b = random_reference(N, 11)
    x = t.solve_inplace(b.copy())
    assert np.linalg.norm(b - t.spmv(x)) / np.linalg.norm(b) < 1e-12
    assert _relerr(x, o.solve_inplace(b)) < 1e-12


@pytest.mark.parametrize("kind,n,d,L,tol,skip", [
    ("lapl", 64, 2, 6, 1e-2, 0),
    ("lapl", 64, 2, 6, 1e-2, 1),
    ("lapl", 32, 3, 8, 1e-2, 0),
    ("diff", 16, 3, 6, 1e-2, 0),
    ("chan", 16, 3, 6, 1e-2, 0),
    ("convdiff", 64, 2, 6, 1e-2, 0),
    ("lapl", 32, 2, 5, 1e-1, 0),
])
def test_factor_and_solve_parity(kind, n, d, L, tol, skip):
    t, o = _pair(kind, n, d, L, tol, skip)
    oc, tc = o.clusters(), t.clusters()
    assert [c["rank"] for c in oc] == [c["rank"] for c in tc]
    # R blocks of the level-0 interiors, and of the top separator
    for q, c in enumerate(oc):
        if c["merge_lvl"] == 0 and c["lvl"] == 0:
            Ro, Rt = np.triu(o.block(q, q)), np.triu(t.block(q, q))
            assert np.abs(Ro - Rt).max() <= RTOL * np.abs(Ro).max()
    top = o.level(L - 1)[0][0]
    Ro, Rt = np.triu(o.block(top, top)), np.triu(t.block(top, top))
    assert np.abs(Ro - Rt).max() <= 1e-9 * np.abs(Ro).max()
    # sparsification reflectors
    for q, c in enumerate(oc):
        if c["sparsified"]:
            Vo, _ = o.qsp(q)
            Vt = t.factor(q, 2)
            assert Vo.shape == Vt.shape
            np.testing.assert_allclose(np.tril(Vt, -1), np.tril(Vo, -1), rtol=0, atol=1e-9)
    N = n ** d
    b = random_reference(N, 2021)
    xo = o.solve_inplace(b)
    xt = t.solve_inplace(b.copy())
    assert _relerr(xt, xo) < 1e-9
    xg = b.copy()
    k, rr = dist_gmres(None, xg, t, 300, 1e-12)
    _, ko, rro, _ = o.gmres(b.copy(), 300, 1e-12)
    assert k == ko
    assert rr < 1e-10


@pytest.mark.parametrize("name,case", [
    ("lapl2d_16_l3", (16, 2, 3, 1e-2, 0)),
    ("lapl2d_64_l6", (64, 2, 6, 1e-2, 0)),
    ("lapl2d_64_l6_skip1", (64, 2, 6, 1e-2, 1)),
    ("lapl3d_16_l6", (16, 3, 6, 1e-2, 0)),
])
def test_against_golden_fixtures(name, case):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    n, d, L, tol, skip = case
    cp, ri, v = M.laplacian(n, d)
    t = ParTree(L, skip)
    t.set_tol(tol)
    t.set_coords_tensor(n, d)
    t.partition((cp, ri, scale_columns(cp, v)))
    t.assemble()
    t.factorize()
    assert np.array_equal(t.perm(), g["perm"])
    assert np.array_equal(np.array([c["rank"] for c in t.clusters()]), g["rank"])
    top = t.level_range(L - 1)[0]
    np.testing.assert_allclose(np.abs(np.diag(t.block(top, top))), g["top_rdiag"], rtol=1e-9)
    b = random_reference(n ** d, 2021)
    x = t.solve_inplace(b.copy())
    assert _relerr(x, g["precond_x"]) < 1e-9
    k, rr = dist_gmres(None, b.copy(), t, 300, 1e-12)
    assert k == int(g["gmres_iters"])
    assert rr < 1e-10


def test_global_solve_matches_permuted_solve():
    n, d, L = 32, 2, 5
    cp, ri, v = M.laplacian(n, d)
    t = ParTree(L, 0)
    t.set_tol(1e-2)
    t.set_coords_tensor(n, d)
    t.partition((cp, ri, scale_columns(cp, v)))
    t.assemble()
    t.factorize()
    b = random_reference(n * n, 5)
    xg = t.solve(b)
    bl = np.zeros(n * n)
    t.distribute_x(b, bl)
    xl = t.solve_inplace(bl)
    np.testing.assert_allclose(xg, t.extract_x(xl), rtol=0, atol=0)


def test_gmres_64cube_manufactured_solution():
    """Full-size property: A x = b with a known x is solved to the requested residual."""
    n, d, L = 64, 3, 12
    cp, ri, v = M.laplacian(n, d)
    t = ParTree(L, 0)
    t.set_tol(1e-2)
    t.set_coords_tensor(n, d)
    t.partition((cp, ri, scale_columns(cp, v)))
    t.assemble()
    t.factorize()
    N = n ** d
    x_true = np.random.default_rng(0).standard_normal(N)
    b = t.spmv(x_true)
    x = b.copy()
    k, rr = dist_gmres(None, x, t, 100, 1e-12)
    assert rr < 1e-10
    assert k <= 20
    assert _relerr(x, x_true) < 1e-6


def test_reassembly_is_bit_identical():
    """A second assemble of the same partition reuses the nonzeros' block maps
    and the CSR permutation built by the first: the factors, the preconditioner
    apply and the GMRES solve are bit-identical, in FP64 and in float storage
    (which rebuilds the maps for the float layout)."""
    cp, ri, v = _matrix("diff", 16, 3)
    t = ParTree(6, 0)
    t.set_tol(1e-2)
    t.set_coords_tensor(16, 3)
    t.partition((cp, ri, scale_columns(cp, v)))
    b = random_reference(16 ** 3, 9)
    t.set_tensor_cores(1)  # one fixed kind of float apply (the tuned mode measures both first)
    for prec in (64, 32, 64):
        t.set_precision(prec)
        out = []
        for _ in range(2):
            t.assemble()
            t.factorize()
            top = len(t.clusters()) - 1
            x = t.solve_inplace(b.copy())
            k, rr = dist_gmres(None, b.copy(), t, 100, 1e-10)
            out.append((t.block(top, top), x, k, rr, [c["rank"] for c in t.clusters()]))
        (B0, x0, k0, r0, rk0), (B1, x1, k1, r1, rk1) = out
        assert rk0 == rk1 and k0 == k1 and r0 == r1
        assert np.array_equal(B0, B1) and np.array_equal(x0, x1)
        assert r0 <= 1e-10


@pytest.mark.parametrize("precision,learned", [(64, False), (32, True)])
def test_reused_plans_are_bit_identical(precision, learned):
    """A re-factorization that meets the same sizes reuses every level's
    descriptor lists; its factors, apply and GMRES are bit-identical to a
    factorization that rebuilds them.  A new tolerance changes the kept ranks:
    the levels above the first changed rank rebuild their lists, and the result
    equals an uncached factorization at that tolerance."""
    from pspaqr_public_b200.tree import load_rank_model

    cp, ri, v = _matrix("diff", 16, 3)
    b = random_reference(16 ** 3, 9)

    def run(cache, tol, reps):
        t = ParTree(6, 0)
        t.set_tol(tol[0] if isinstance(tol, list) else tol)
        t.set_tensor_cores(1)
        t.set_coords_tensor(16, 3)
        t.set_precision(precision)
        t.set_plan_cache(cache)
        t.partition((cp, ri, scale_columns(cp, v)))
        if learned:
            t.set_rank_model(load_rank_model(), 32)
        outs = []
        for tol_i in tol if isinstance(tol, list) else [tol] * reps:
            t.set_tol(tol_i)
            t.assemble()
            t.factorize()
            top = len(t.clusters()) - 1
            x = t.solve_inplace(b.copy())
            k, rr = dist_gmres(None, b.copy(), t, 100, 1e-10)
            outs.append((t.block(top, top), x, k, rr, [c["rank"] for c in t.clusters()]))
        return t, outs

    t, cached = run(True, 1e-2, 3)
    assert t.plan_hits() == 2 * 6  # every level of the 2nd and 3rd factorization
    _, fresh = run(False, 1e-2, 1)
    for B, x, k, rr, rk in cached:
        B0, x0, k0, rr0, rk0 = fresh[0]
        assert rk == rk0 and k == k0 and rr == rr0
        assert np.array_equal(B, B0) and np.array_equal(x, x0)
    t2, mixed = run(True, [1e-2, 1e-3], 0)
    assert t2.plan_hits() < 6
    _, fresh3 = run(False, 1e-3, 1)
    B, x, k, rr, rk = mixed[1]
    B0, x0, k0, rr0, rk0 = fresh3[0]
    assert rk == rk0 and k == k0 and np.array_equal(B, B0) and np.array_equal(x, x0)


def test_tuned_applies_pick_the_faster_kind_per_level():
    """Mode 2 (the default): the first float factorization runs every apply on the
    tensor cores, the second on the CUDA cores; later ones use, per level and kind
    of apply, the one measured faster.  Every one of them is a valid factor."""
    cp, ri, v = _matrix("diff", 16, 3)
    t = ParTree(6, 0)
    t.set_tol(1e-2)
    t.set_coords_tensor(16, 3)
    t.set_precision(32)
    t.partition((cp, ri, scale_columns(cp, v)))
    b = random_reference(16 ** 3, 4)
    etas = []
    for _ in range(3):
        t.assemble()
        t.factorize()
        etas.append(t.backward_error(2, seed=5))
        k, rr = dist_gmres(None, b.copy(), t, 100, 1e-10)
        assert rr <= 1e-10
    tab = t.tune_table()
    measured = tab[:, :, 0] >= 0
    assert measured.any()
    for l, k in zip(*np.nonzero(measured)):
        # the tensor cores where they were at least 5 % faster, else the CUDA cores
        assert tab[l, k, 2] == (1.0 if tab[l, k, 0] < np.float32(0.95) * tab[l, k, 1] else 0.0)
    assert np.all(np.abs(np.array(etas) / etas[1] - 1) < 0.2)
