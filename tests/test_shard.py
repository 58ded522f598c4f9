"""Subtree sharding over ranks (pspaqr_public_b200.shard), on the host.

* The plan restates cluster2rank / edge2rank (ptree.cpp:65-91): leaf sections
  block-distributed, the top levels on fewer ranks, every transfer between
  ranks (factors, compression blocks, merged blocks) listed once with the right
  sender and receiver.
* Two gloo ranks (world size 2, CPU): the owned clusters partition the tree, every
  level's exchange delivers exactly the payloads each rank must receive, and
  flexible GMRES over the sharded vectors (dots by all-reduce, the SpMV with a
  halo exchange) reproduces the single-rank run: same iteration count, the same
  solution to 1e-10.  No GPU: the operator is the partitioned matrix itself
  with a Jacobi preconditioner, standing in for the per-rank factor apply.
"""
import json
import os
import socket

import numpy as np
import pytest
import scipy.sparse as sp

from pspaqr_public_b200 import ParTree, scale_columns
from pspaqr_public_b200 import matrices as M
from pspaqr_public_b200.shard import ShardPlan, dist_fgmres

N, D, L = 16, 3, 6


def _tree():
    cp, ri, v = M.diffusion_lognormal(N, D, seed=2)
    vs = scale_columns(cp, v)
    t = ParTree(L, 0)
    t.set_tol(1e-2)
    t.set_coords_tensor(N, D)
    t.partition((cp, ri, vs))
    A = sp.csc_matrix((vs, ri, cp), shape=(N ** D, N ** D))
    p = t.perm()
    return t, sp.csr_matrix(A[p][:, p])


@pytest.mark.parametrize("nranks", [1, 2, 4, 8])
def test_plan_restates_cluster2rank(nranks):
    t, _ = _tree()
    plan = ShardPlan(t, nranks)
    cl = t.clusters()
    nparts = 2 ** (L - 1)
    for o, c in enumerate(cl):
        parts = nparts >> c["merge_lvl"]
        want = c["section"] // (parts // nranks) if parts > nranks else c["section"]
        assert plan.cluster_owner[o] == want
    assert plan.cluster_owner[-1] == 0  # the root
    counts = np.bincount(plan.row_owner, minlength=nranks)
    assert counts.min() > 0 and counts.max() <= 1.5 * counts.mean()
    for lvl, ex in enumerate(plan.exchange):
        for kind, idx, dst, frm, to in ex.tolist():
            assert frm != to and 0 <= frm < nranks and 0 <= to < nranks
            if kind == 0:  # merge: child block of this level into a parent block of the next
                assert plan.edge_owner[idx] == frm and plan.edge_owner[dst] == to
                assert plan.edges[idx, 2] == lvl and plan.edges[dst, 2] == lvl + 1
            elif kind == 3:  # compression gather: block A(p, m) to the owner of p
                assert plan.edge_owner[idx] == frm and plan.cluster_owner[plan.edges[idx, 1]] == to
            else:  # factors of a cluster of this level
                assert plan.cluster_owner[idx] == frm and cl[idx]["merge_lvl"] == lvl
    total = sum(len(e) for e in plan.exchange)
    if nranks == 1:
        assert total == 0
    else:
        assert total > 0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _block(edge, rows, cols):
    return np.arange(rows * cols, dtype=np.float64).reshape(rows, cols) + 1000.0 * edge


def _rank_main(rank, world, port, outdir):
    import torch.distributed as dist

    from pspaqr_public_b200.shard import exchange

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t, A = _tree()
        plan = ShardPlan(t, world)
        sizes = np.array([c["size_org"] for c in t.clusters()])
        out = {"owned": np.flatnonzero(plan.cluster_owner == rank).tolist(), "received_ok": True, "nrecv": 0}
        # every level's transfers with payloads of their pre-compression sizes
        def payload(kind, idx):
            if kind in (0, 3):
                return _block(idx, sizes[plan.edges[idx, 1]], sizes[plan.edges[idx, 0]])
            return _block(idx, sizes[idx], sizes[idx])

        for lvl in range(L):
            got = exchange(plan, lvl, rank, payload)
            want = {(k, i) for k, i, _, _, to in plan.exchange[lvl].tolist() if to == rank}
            out["received_ok"] &= set(got) == want
            for (k, i), a in got.items():
                out["received_ok"] &= bool(np.array_equal(a, payload(k, i)))
            out["nrecv"] += len(got)
        # flexible GMRES over the sharded unknowns
        rows = plan.owned_rows(rank)
        n = A.shape[0]
        A_loc = A[rows]
        dinv = 1.0 / A.diagonal()[rows]

        def apply_A(x_loc):
            import torch

            full = torch.zeros(n, dtype=torch.float64)
            full[rows] = torch.from_numpy(x_loc)
            dist.all_reduce(full)  # the halo: every rank's owned entries
            return A_loc @ full.numpy()

        b = np.random.default_rng(5).standard_normal(n)
        x_loc, k, rr = dist_fgmres(apply_A, lambda v: dinv * v, b[rows].copy(), 200, 1e-10)
        out.update(k=k, relres=rr, rows=rows.tolist(), x=x_loc.tolist())
        with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
            json.dump(out, f)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    t, A = _tree()
    owned = sorted(res[0]["owned"] + res[1]["owned"])
    assert owned == list(range(t.num_clusters())) and not set(res[0]["owned"]) & set(res[1]["owned"])
    assert all(r["received_ok"] for r in res) and sum(r["nrecv"] for r in res) > 0
    # single-rank reference run of the same Krylov code
    n = A.shape[0]
    b = np.random.default_rng(5).standard_normal(n)
    dinv = 1.0 / A.diagonal()
    x1, k1, rr1 = dist_fgmres(lambda x: A @ x, lambda v: dinv * v, b.copy(), 200, 1e-10)
    assert res[0]["k"] == res[1]["k"] == k1
    x = np.zeros(n)
    for r in res:
        x[np.array(r["rows"], dtype=int)] = r["x"]
    assert np.linalg.norm(x - x1) <= 1e-10 * np.linalg.norm(x1)
    assert max(r["relres"] for r in res) <= 1e-9
