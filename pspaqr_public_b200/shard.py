"""Nested-dissection subtree sharding over ranks (one GPU per rank).

The reference distributes ParTree over MPI ranks by subtree: ``cluster2rank``
(ptree.cpp:65-91) gives each leaf section and the clusters above it an owner,
blocks live with the owner of their column cluster, the blocks whose parent
block has another owner are sent when a level is merged into the next
(``send_edge_am``, ptree.cpp:2005-2038), and GMRES reduces its dots and norms
with ``MPI_Allreduce`` (``VecDot`` / ``VecNorm``, util.cpp:1052-1066).

This module holds the host side of that split for ``torch.distributed``
(NCCL between GPUs, gloo on the host):

* :class:`ShardPlan` -- the owners and the per-level exchange lists, computed by
  the library from the partition (``spq_shard_plan`` / ``spq_shard_exchange``);
* :func:`exchange` -- one level's transfers (factors to the owners of the
  blocks they update, compression blocks to their interface's owner, blocks
  merged into a parent owned elsewhere) as point-to-point messages;
* :func:`dist_dot` and :func:`dist_fgmres` -- flexible GMRES over vectors sharded
  by ``ShardPlan.row_owner``, every inner product an all-reduce.

The factorization kernels themselves still run on one GPU (``ParTree``); the
plan and the distributed Krylov layer are what a per-rank factorization of the
owned subtrees plugs into.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Dict, List, Optional

import numpy as np

from .tree import ParTree, lib


class ShardPlan:
    """Owners of clusters, unknowns and blocks for ``nranks`` ranks, and the blocks
    that cross ranks at each level's merge."""

    def __init__(self, tree: ParTree, nranks: int):
        self.nranks = nranks
        ncl = tree.num_clusters()
        n = tree.nrows_local()
        L = tree.nlevels
        self.cluster_owner = np.zeros(ncl, np.int32)
        self.row_owner = np.zeros(n, np.int32)
        nex = np.zeros(L, np.int32)
        tree._chk(lib().spq_shard_plan(tree._h, nranks, _pi(self.cluster_owner), _pi(self.row_owner), _pi(nex)),
                  "shard_plan")
        # per level: (kind, id, dst, from, to) rows, kinds as spq_shard_exchange
        self.exchange: List[np.ndarray] = []
        for lvl in range(L):
            out = np.zeros(5 * max(int(nex[lvl]), 1), np.int32)
            tree._chk(lib().spq_shard_exchange(tree._h, nranks, lvl, _pi(out)), "shard_exchange")
            self.exchange.append(out[: 5 * int(nex[lvl])].reshape(-1, 5))
        ne = tree.num_edges()
        e = np.zeros(3 * max(ne, 1), np.int32)
        tree._chk(lib().spq_get_edges(tree._h, _pi(e)), "get_edges")
        self.edges = e[: 3 * ne].reshape(ne, 3)  # n1 (column cluster), n2 (row cluster), level
        self.edge_owner = self.cluster_owner[self.edges[:, 0]]

    def owned_rows(self, rank: int) -> np.ndarray:
        """Permuted unknowns owned by ``rank`` (ascending)."""
        return np.flatnonzero(self.row_owner == rank)


def _pi(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


KIND_MERGE, KIND_ELIM_FACTORS, KIND_IFACE_FACTORS, KIND_GATHER = 0, 1, 2, 3


def exchange(plan: ShardPlan, lvl: int, rank: int, payload: Callable[[int, int], np.ndarray]) -> Dict[tuple, np.ndarray]:
    """One level's transfers between ranks as point-to-point messages: this rank
    sends ``payload(kind, id)`` for every transfer it originates and receives the
    ones addressed to it, returned as {(kind, id): array}.  Every rank walks the
    level's list in the same order, so sends and receives pair up without tags
    and without deadlock (a blocking send waits only for a receive that the
    destination reaches before any later transfer)."""
    import torch
    import torch.distributed as dist

    received = {}
    for kind, idx, _, frm, to in plan.exchange[lvl].tolist():
        if frm == rank:
            a = np.ascontiguousarray(payload(kind, idx), dtype=np.float64)
            a2 = a.reshape(a.shape[0], -1) if a.ndim else a.reshape(1, 1)
            head = torch.tensor([kind, idx, a2.shape[0], a2.shape[1]], dtype=torch.int64)
            dist.send(head, dst=to)
            if a2.size:
                dist.send(torch.from_numpy(a2.ravel().copy()), dst=to)
        elif to == rank:
            head = torch.zeros(4, dtype=torch.int64)
            dist.recv(head, src=frm)
            r, c = int(head[2]), int(head[3])
            buf = torch.zeros(r * c, dtype=torch.float64)
            if r * c:
                dist.recv(buf, src=frm)
            received[(int(head[0]), int(head[1]))] = buf.numpy().reshape(r, c)
    return received


def dist_dot(x: np.ndarray, y: np.ndarray) -> float:
    """VecDot (util.cpp:1058-1066): the local dot of the owned entries, summed
    over ranks by an all-reduce."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(np.dot(x, y))], dtype=torch.float64)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t)
    return float(t[0])


def dist_fgmres(apply_A: Callable[[np.ndarray], np.ndarray], apply_M: Callable[[np.ndarray], np.ndarray],
                b: np.ndarray, maxit: int = 300, tol: float = 1e-10, hist: Optional[list] = None):
    """Flexible right-preconditioned GMRES (x0 = 0) over sharded vectors.

    ``b`` holds this rank's owned entries; ``apply_A`` and ``apply_M`` map owned
    entries to owned entries (each does its own halo exchange).  Every inner
    product and norm is a :func:`dist_dot` all-reduce, so all ranks take the same
    Givens rotations and stop at the same step.  Returns ``(x, k, relres)`` with
    the true ||b - A x|| / ||b||; k is the 0-based step of the break, as in
    is.cpp:447-527.
    """
    n = b.size
    bn = np.sqrt(dist_dot(b, b))
    V = np.zeros((maxit + 1, n))
    Z = np.zeros((maxit, n))
    H = np.zeros((maxit + 1, maxit))
    cs, sn = np.zeros(maxit), np.zeros(maxit)
    beta = np.zeros(maxit + 1)
    V[0] = b / bn
    beta[0] = bn
    k = 0
    for k in range(maxit):
        Z[k] = apply_M(V[k])
        w = apply_A(Z[k])
        for i in range(k + 1):  # modified Gram-Schmidt, one all-reduce per dot
            H[i, k] = dist_dot(w, V[i])
            w = w - H[i, k] * V[i]
        H[k + 1, k] = np.sqrt(dist_dot(w, w))
        V[k + 1] = w / H[k + 1, k] if H[k + 1, k] != 0 else w
        for i in range(k):
            t = cs[i] * H[i, k] + sn[i] * H[i + 1, k]
            H[i + 1, k] = -sn[i] * H[i, k] + cs[i] * H[i + 1, k]
            H[i, k] = t
        r = np.hypot(H[k, k], H[k + 1, k])
        cs[k], sn[k] = (H[k, k] / r, H[k + 1, k] / r) if r != 0 else (1.0, 0.0)
        H[k, k] = r
        H[k + 1, k] = 0.0
        beta[k + 1] = -sn[k] * beta[k]
        beta[k] = cs[k] * beta[k]
        err = abs(beta[k + 1]) / bn
        if hist is not None:
            hist.append(err)
        if err <= tol:
            break
    m = k + 1
    y = np.linalg.solve(np.triu(H[:m, :m]), beta[:m])
    x = Z[:m].T @ y
    r = b - apply_A(x)
    return x, k, float(np.sqrt(dist_dot(r, r)) / bn)
