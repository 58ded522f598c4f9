"""GPU path against the oracle's 64^3 fixtures (tests/golden/*_64_*.npz, written by
make_golden_64.py): the size the headline workload runs at.

Plain FP64 (the reference method): permutation, every kept rank and the GMRES
iteration counts exact; the top separator's |diag R|, the preconditioner apply of
the reference right-hand side and the factor backward error within 1e-9 relative
(summation order is the only difference from LAPACK).  Vectors are compared through
the fixtures' summaries (4096 seeded entries, the norm and 8 seeded projections):
an error e with ||e|| <= 1e-9 ||x|| moves each summary by at most about 1e-9 ||x||.

Mixed precision (float factors, 3xTF32 tensor-core trailing updates, FP64 Krylov):
checked against the same FP64 oracle -- kept ranks, the factor backward error, and
the true residual of flexible GMRES, which must reach 1e-10.
"""
import hashlib
import os

import numpy as np
import pytest

from pspaqr_public_b200 import ParTree, dist_gmres, random_reference, scale_columns
from pspaqr_public_b200 import matrices as M

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
N_SAMPLES, N_PROJ, N_PROBES = 4096, 8, 3

CASES = {
    "lapl3d_64_t1e-2": ("lapl", 1e-2, 1),
    "diff3d_64_t1e-2": ("diff", 1e-2, 2),
    "diff3d_64_t1e-3": ("diff", 1e-3, 2),
}

_mats = {}


def _matrix(kind):
    if kind not in _mats:
        _mats[kind] = M.laplacian(64, 3) if kind == "lapl" else M.diffusion_lognormal(64, 3, seed=2)
    return _mats[kind]


def _tree(kind, tol, precision=64):
    cp, ri, v = _matrix(kind)
    t = ParTree(12, 0)
    t.set_tol(tol)
    t.set_coords_tensor(64, 3)
    t.set_precision(precision)
    t.partition((cp, ri, scale_columns(cp, v)))
    t.assemble()
    t.factorize()
    return t


def _summary(x):
    n = x.size
    idx = np.sort(np.random.default_rng(777).choice(n, N_SAMPLES, replace=False))
    P = np.random.default_rng(778).standard_normal((N_PROJ, n)) / np.sqrt(n)
    return x[idx], np.linalg.norm(x), P @ x


def _check_summary(x, g, key, rtol):
    s, nrm, proj = _summary(x)
    ref = float(g[key + "_norm"])
    assert abs(nrm - ref) <= rtol * ref, (key, nrm, ref)
    assert np.abs(s - g[key + "_samples"]).max() <= rtol * ref, key
    assert np.abs(proj - g[key + "_proj"]).max() <= rtol * ref, key


def _probes(n):
    return np.stack([np.random.default_rng(9000 + p).standard_normal(n) for p in range(N_PROBES)], axis=1)


@pytest.mark.parametrize("name", list(CASES))
def test_fp64_matches_oracle_at_64cube(name):
    kind, tol, seed = CASES[name]
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    t = _tree(kind, tol)
    N = 64 ** 3
    assert hashlib.sha256(t.perm().astype(np.int32).tobytes()).hexdigest() == str(g["perm_sha256"])
    ranks = np.array([c["rank"] for c in t.clusters()])
    assert ranks.shape == g["rank"].shape
    bad = np.flatnonzero(ranks != g["rank"])
    assert bad.size == 0, f"{bad.size} kept ranks differ, first at cluster {bad[:5]}"
    top = t.level_range(11)[0]
    np.testing.assert_allclose(np.abs(np.diag(t.block(top, top))), g["top_rdiag"], rtol=1e-9,
                               atol=1e-12 * g["top_rdiag"].max())
    b = random_reference(N, 2021)
    _check_summary(t.solve_inplace(b.copy()), g, "precond_x", 1e-9)
    k, rr = dist_gmres(None, b.copy(), t, 300, 1e-10)
    assert k == int(g["gmres_iters"])
    bn = M.rhs_normal(N, seed)
    xn = bn.copy()
    kn, rrn = dist_gmres(None, xn, t, 300, 1e-10)
    assert kn == int(g["gmres_iters_normal"])
    assert rrn <= 2 * float(g["gmres_relres_normal"]) + 1e-12
    _check_summary(xn, g, "gmres_x_normal", 1e-8)
    eta = t.backward_error(N_PROBES, _probes(N))
    np.testing.assert_allclose(eta, g["backward_error"], rtol=1e-9)


@pytest.mark.parametrize("name", list(CASES))
def test_mixed_precision_against_fp64_oracle_at_64cube(name):
    """Float factors (tensor-core trailing updates): the kept ranks stay those of the
    FP64 oracle on almost every interface, the backward error of the factor stays at
    the oracle's (the sparsification tolerance dominates the float rounding), and
    flexible GMRES in FP64 still reaches a true residual of 1e-10."""
    kind, tol, seed = CASES[name]
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    t = _tree(kind, tol, precision=32)
    N = 64 ** 3
    ranks = np.array([c["rank"] for c in t.clusters()])
    sp = g["sparsified"].astype(bool)
    d = np.abs(ranks[sp] - g["rank"][sp])
    assert np.mean(d == 0) >= 0.97, np.mean(d == 0)
    assert np.mean(d <= 2) >= 0.995, np.mean(d <= 2)
    eta = t.backward_error(N_PROBES, _probes(N))
    ratio = eta / g["backward_error"]
    assert np.all(ratio < 1.25) and np.all(ratio > 0.8), ratio
    x = M.rhs_normal(N, seed)
    k, rr = dist_gmres(None, x, t, 300, 1e-10)
    assert rr <= 1e-10
    assert k <= int(g["gmres_iters_normal"]) + 2
