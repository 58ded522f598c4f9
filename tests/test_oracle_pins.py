"""The CPU oracle against the structural pins and the committed golden fixtures.

The reference publishes no outputs; its partition is pinned by the cluster
counts of a replica of the reference partition (partition.cpp:241-350,
514-587; tree.cpp:48-57; ptree.cpp:587-691) and the oracle's own numerics by
fixtures generated with tests/golden/make_golden.py.
"""
import os

import numpy as np
import pytest

from oracle.oracle import OracleTree, random_reference
from pspaqr_public_b200 import matrices as M

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _oracle(n, d, L, tol=1e-2, skip=0, threads=1, factorize=False):
    cp, ri, v = M.laplacian(n, d)
    o = OracleTree(L, skip, tol, threads)
    o.set_matrix(cp, ri, v)
    o.set_coords_tensor(n, d)
    o.partition()
    o.assemble()
    if factorize:
        o.factorize()
    return o


def _level_table(o, L):
    cls = o.clusters()
    rows = []
    for lvl in range(L):
        orders, ni, nf = o.level(lvl)
        ints = [cls[q]["cols"] for q in orders if cls[q]["lvl"] == lvl]
        itf = [cls[q]["cols"] for q in orders if cls[q]["lvl"] > lvl]
        rows.append((ni, float(np.median(ints)) if ints else None, nf, float(np.median(itf)) if itf else None,
                     max(itf) if itf else None))
    return rows


def test_partition_pin_64x64_5pt():
    L = 6
    o = _oracle(64, 2, L)
    table = _level_table(o, L)
    expect = [(32, 94, 79, 14, 30), (16, 29, 33, 28, 30), (8, 29, 15, 30, 62), (4, 62, 5, 62, 62),
              (2, 62, 1, 128, 128), (1, 128, 0, None, None)]
    assert table == [tuple(e) for e in expect]
    assert len(o.level(0)[0]) == 111
    assert len(o.edges()) == 523


def test_partition_pin_64cube_7pt():
    L = 12
    o = _oracle(64, 3, L)
    table = _level_table(o, L)
    expect = [(2048, 30, 11847, 18, 42), (1024, 28, 5781, 28, 98), (512, 70, 2520, 55, 98), (256, 72, 1193, 70, 210),
              (128, 188, 577, 150, 450), (64, 420, 252, 392, 450), (32, 420, 113, 420, 930), (16, 899, 49, 868, 1922),
              (8, 1922, 18, 1922, 1922), (4, 1922, 5, 3968, 3968), (2, 3968, 1, 8192, 8192), (1, 8192, 0, None, None)]
    assert table == [tuple(e) for e in expect]
    assert len(o.level(0)[0]) == 13895
    assert len(o.edges()) == 105291
    cls = o.clusters()
    # interfaces whose two sides are eliminated below the top two levels (want_sparsify, ptree.cpp:29-41)
    spars = []
    for lvl in range(L):
        orders, _, _ = o.level(lvl)
        spars.append(sum(1 for q in orders if cls[q]["lvl"] > lvl and cls[q]["l_lvl"] <= lvl
                         and cls[q]["r_lvl"] <= lvl and lvl < L - 2))
    assert spars == [6222, 3057, 1344, 670, 325, 144, 70, 31, 12, 4, 0, 0]


@pytest.mark.parametrize("name,case", [
    ("lapl2d_16_l3", (16, 2, 3, 1e-2, 0)),
    ("lapl2d_64_l6", (64, 2, 6, 1e-2, 0)),
    ("lapl2d_64_l6_skip1", (64, 2, 6, 1e-2, 1)),
    ("lapl3d_16_l6", (16, 3, 6, 1e-2, 0)),
])
def test_oracle_matches_golden(name, case):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    n, d, L, tol, skip = case
    o = _oracle(n, d, L, tol, skip, factorize=True)
    cls = o.clusters()
    assert np.array_equal(o.perm(), g["perm"])
    assert np.array_equal(np.array([c["rank"] for c in cls]), g["rank"])
    top = o.level(L - 1)[0][0]
    np.testing.assert_allclose(np.abs(np.diag(o.block(top, top))), g["top_rdiag"], rtol=1e-12)
    b = random_reference(n ** d, 2021)
    x = o.solve_inplace(b)
    np.testing.assert_allclose(x, g["precond_x"], rtol=1e-12, atol=1e-12 * np.abs(g["precond_x"]).max())
    _, k, rr, _ = o.gmres(b.copy(), 300, 1e-12)
    assert k == int(g["gmres_iters"])
    assert rr < 1e-10


def test_oracle_exact_without_sparsification():
    """tol = 0 keeps every rank: the factorization is an exact QR (residual ~ eps)."""
    o = _oracle(16, 2, 4, tol=0.0, factorize=True)
    b = random_reference(256, 7)
    x = o.solve_inplace(b)
    assert np.linalg.norm(b - o.spmv(x)) / np.linalg.norm(b) < 1e-13
    o3 = _oracle(8, 3, 4, tol=0.0, factorize=True)
    b3 = random_reference(512, 9)
    x3 = o3.solve_inplace(b3)
    assert np.linalg.norm(b3 - o3.spmv(x3)) / np.linalg.norm(b3) < 1e-13


def test_oracle_thread_count_is_bitwise_invariant():
    a = _oracle(32, 2, 5, threads=1, factorize=True)
    b = _oracle(32, 2, 5, threads=4, factorize=True)
    v = random_reference(1024, 3)
    assert np.array_equal(a.solve_inplace(v), b.solve_inplace(v))
    assert [c["rank"] for c in a.clusters()] == [c["rank"] for c in b.clusters()]


def test_reference_rhs_generator():
    """mt19937 + U(-1,1) (util.cpp:992-1001): first draws of seed 2021 are stable."""
    x = random_reference(5, 2021)
    assert np.all(np.abs(x) <= 1.0)
    np.testing.assert_array_equal(x, random_reference(5, 2021))
    assert not np.array_equal(x, random_reference(5, 2022))


def test_tie_rule_keeps_lapack_observables():
    """The oracle's restated dlaqp2 with the tie-tolerant pivot keeps the kept
    ranks and the GMRES iteration count of LAPACK's dgeqp3 (the call the
    reference makes, ptree.cpp:405-414); only which of several equal-norm
    columns is pivoted first can differ."""
    res = {}
    for mode in (0, 1):
        cp, ri, v = M.laplacian(64, 2)
        o = OracleTree(6, 0, 1e-2, 1)
        o.set_pivot(mode, 1e-6)
        o.set_matrix(cp, ri, v)
        o.set_coords_tensor(64, 2)
        o.partition()
        o.assemble()
        o.factorize()
        b = random_reference(4096, 2021)
        _, k, rr, _ = o.gmres(b, 300, 1e-12)
        res[mode] = ([c["rank"] for c in o.clusters()], k, rr)
    assert res[0][0] == res[1][0]
    assert res[0][1] == res[1][1]
    assert res[0][2] < 1e-11 and res[1][2] < 1e-11
