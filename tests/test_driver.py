"""The spaqr command-line driver (pspaQR.cpp's options and report lines)."""
import os
import re
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "pspaqr_public_b200", "spaqr")


def _run(*args):
    return subprocess.run([DRIVER, *args], capture_output=True, text=True, timeout=600)


def test_help_and_mandatory_matrix():
    r = _run("--help")
    assert r.returncode == 0 and "--matrix" in r.stdout and "--res" in r.stdout
    r = _run()
    assert r.returncode == 0 and "--matrix is mandatory" in r.stdout
    r = _run("-m", "x.mtx", "--coordinates", "c.mtx")
    assert r.returncode == 1 and "not supported" in r.stderr


def _write_mm(path, A):
    A = sp.coo_matrix(A)
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{A.shape[0]} {A.shape[1]} {A.nnz}\n")
        for i, j, v in zip(A.row, A.col, A.data):
            f.write(f"{i + 1} {j + 1} {v:.17g}\n")


@pytest.mark.gpu
def test_driver_solves_like_the_python_api(tmp_path):
    from pspaqr_public_b200 import ParTree, dist_gmres, random_reference, scale_columns
    from pspaqr_public_b200 import matrices as M

    n = 32
    cp, ri, v = M.laplacian(n, 2)
    A = sp.csc_matrix((v, ri, cp), shape=(n * n, n * n))
    path = str(tmp_path / "lapl.mtx")
    _write_mm(path, A)
    r = _run("-m", path, "-n", str(n), "-d", "2", "-l", "5", "-t", "1e-2", "-i", "100", "--res", "1e-12")
    assert r.returncode == 0, r.stderr
    out = r.stdout
    assert "Matrix " + path in out and "Time to factorize:" in out
    one = float(re.search(r"<<<<\|\(Ax-b\)\|/\|b\| : (\S+)", out).group(1))
    m = re.search(r"GMRES: #iterations: (\d+), residual \|Ax-b\|/\|b\|: (\S+)", out)
    k, rr = int(m.group(1)), float(m.group(2))
    assert rr <= 1e-12 and one < 1.0
    t = ParTree(5, 0)
    t.set_tol(1e-2)
    t.set_coords_tensor(n, 2)
    t.partition((cp, ri, scale_columns(cp, v)))
    t.assemble()
    t.factorize()
    k2, rr2 = dist_gmres(None, random_reference(n * n, 2021), t, 100, 1e-12)
    assert k == k2
    assert np.isclose(rr, rr2, rtol=1e-3, atol=1e-15)
