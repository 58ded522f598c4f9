"""Host partition + symbolic structure of the product against the oracle (CPU only).

The ordering must be identical to the reference's (partition.cpp:282-350,
514-587; tree.cpp:48-57): permutation, cluster ids, hierarchy and the block
structure of every level (fill-in ptree.cpp:101-153, merge ptree.cpp:289-340).
"""
import numpy as np
import pytest

from oracle.oracle import OracleTree
from pspaqr_public_b200 import ParTree, SpqError, scale_columns
from pspaqr_public_b200 import matrices as M

CASES = [
    ("lapl", 16, 2, 3),
    ("lapl", 64, 2, 6),
    ("lapl", 32, 2, 7),
    ("lapl", 16, 3, 6),
    ("lapl", 32, 3, 8),
    ("lapl", 8, 3, 2),
    ("convdiff", 32, 2, 5),
    ("diff", 16, 3, 5),
]


def _matrix(kind, n, d):
    if kind == "lapl":
        return M.laplacian(n, d)
    if kind == "convdiff":
        return M.convection_diffusion_2d(n)
    return M.diffusion_lognormal(n, d, seed=5)


@pytest.mark.parametrize("kind,n,d,L", CASES)
def test_partition_identical(kind, n, d, L):
    cp, ri, v = _matrix(kind, n, d)
    vs = scale_columns(cp, v)
    t = ParTree(L, 0)
    t.set_tol(1e-2)
    t.set_coords_tensor(n, d)
    t.partition((cp, ri, vs))
    o = OracleTree(L, 0, 1e-2, 1)
    o.set_matrix(cp, ri, v)
    o.set_coords_tensor(n, d)
    o.partition()
    o.assemble()
    np.testing.assert_array_equal(o.matrix_values(), vs)
    np.testing.assert_array_equal(t.perm(), o.perm())
    oc, tc = o.clusters(), t.clusters()
    assert len(oc) == len(tc)
    for a, b in zip(oc, tc):
        assert (a["lvl"], a["merge_lvl"], a["cols"], a["parent"], a["section"], a["sep"]) == \
            (b["lvl"], b["merge_lvl"], b["size"], b["parent"], b["section"], b["sep"])
        assert (a["l_lvl"], a["l_sep"], a["r_lvl"], a["r_sep"]) == (b["l_lvl"], b["l_sep"], b["r_lvl"], b["r_sep"])
    # every block the oracle creates over the whole factorization exists in the product's symbolic structure
    o.factorize()
    oedges = {(int(a), int(b)) for a, b, _, _ in o.edges()}
    assert t.num_edges() == len(oedges)
    assert all(t.find_edge(a, b) >= 0 for a, b in oedges)


def test_levels_and_ranges():
    cp, ri, v = M.laplacian(64, 2)
    t = ParTree(6, 0)
    t.set_coords_tensor(64, 2)
    t.partition((cp, ri, scale_columns(cp, v)))
    first, count = t.level_range(0)
    assert (first, count) == (0, 111)
    total = sum(t.level_range(l)[1] for l in range(6))
    assert total == t.num_clusters()
    # leaves tile the permuted index range
    cls = t.clusters()
    starts = sorted((c["cstart"], c["size"]) for c in cls[:count])
    pos = 0
    for s, n in starts:
        assert s == pos
        pos += n
    assert pos == 64 * 64


def test_partition_errors():
    cp, ri, v = M.laplacian(8, 2)
    t = ParTree(3, 0)
    with pytest.raises(SpqError):  # no coordinates
        t.partition((cp, ri, v))
    t.set_coords_tensor(9, 2)
    with pytest.raises(SpqError):  # coordinate count mismatch
        t.partition((cp, ri, v))
    with pytest.raises(SpqError):
        ParTree(1, 0)
    t2 = ParTree(3, 0)
    with pytest.raises(SpqError):  # rectangular systems are not built
        t2.set_square(0)
    t3 = ParTree(3, 0)
    t3.set_coords_tensor(8, 2)
    with pytest.raises(SpqError):  # assemble before partition
        t3.assemble()
    with pytest.raises(SpqError):
        t3.factorize()
