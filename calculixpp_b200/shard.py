"""Row-sharded assembly of one model across ranks, with no collective on the data path.

Rank r owns a contiguous range of nodes and therefore (free equations being numbered
in node order) a contiguous range of global rows. It integrates every element incident
to an owned node, the halo elements included, and keeps only the owned rows. A shard
is an ordinary model: the incident elements in ascending global order, the nodes they
use in ascending global order, the global DOF map restricted to those nodes. Both
renumberings are monotone, so every owned row of the shard holds exactly the global
row's columns in the same order, summed over the same elements in the same order as
the single-GPU assembly: the concatenated owned rows equal the global K_ff and rhs.

Node ranges are cut so that the owned rows' non-zero counts are balanced.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .assembly import Model
from .meshgen import Mesh


def node_row_weights(model: Model) -> np.ndarray:
    """Estimated CSR non-zeros of each node's rows: free components x 3 x (nodes sharing
    an element with it); constrained columns are counted too, so it is an upper bound."""
    m = model.mesh
    n = m.conn.shape[1]
    dof_eq, _, _ = model.dof_map()
    free = (dof_eq.reshape(-1, 3) >= 0).sum(1)
    a = np.repeat(m.conn, n, axis=1).reshape(-1).astype(np.int64)
    b = np.tile(m.conn, (1, n)).reshape(-1).astype(np.int64)
    key = np.unique(a * m.n_nodes + b)
    deg = np.bincount(key // m.n_nodes, minlength=m.n_nodes)
    return free * 3 * deg


def partition_nodes(weights: np.ndarray, n_parts: int) -> np.ndarray:
    """Cut points c[0]=0 < ... < c[n_parts]=N of contiguous node ranges with balanced
    total weight."""
    N = weights.size
    if n_parts < 1 or n_parts > max(N, 1):
        raise ValueError("need 1 <= n_parts <= n_nodes")
    cum = np.concatenate([[0], np.cumsum(weights, dtype=np.float64)])
    targets = cum[-1] * np.arange(1, n_parts) / n_parts
    cuts = np.searchsorted(cum, targets, side="left")
    cuts = np.clip(cuts, 1, N - 1) if N > 1 else cuts
    cuts = np.maximum.accumulate(np.concatenate([[0], cuts, [N]]))
    for i in range(1, n_parts + 1):  # keep every range non-empty
        cuts[i] = max(cuts[i], cuts[i - 1] + 1) if i < n_parts else N
    return cuts.astype(np.int64)


@dataclass
class Shard:
    """One rank's part: `model` is the shard model; rows [row0, row0 + n_rows) of the
    global system are its local rows [local_row0, local_row0 + n_rows); the global
    equation of local equation j is eq_global[j]; nodes[k] is the global id of local
    node k and elems[k] of local element k."""

    rank: int
    node_range: tuple
    model: Model
    nodes: np.ndarray
    elems: np.ndarray
    eq_global: np.ndarray
    row0: int
    n_rows: int
    local_row0: int


def make_shard(model: Model, cuts: np.ndarray, rank: int) -> Shard:
    m = model.mesh
    n0, n1 = int(cuts[rank]), int(cuts[rank + 1])
    owned = (m.conn >= n0) & (m.conn < n1)
    elems = np.nonzero(owned.any(axis=1))[0]
    conn_g = m.conn[elems]
    nodes = np.unique(conn_g)
    local = np.full(m.n_nodes, -1, dtype=np.int64)
    local[nodes] = np.arange(nodes.size)
    sub = Mesh(coords=np.ascontiguousarray(m.coords[nodes]), conn=np.ascontiguousarray(local[conn_g], dtype=np.int32),
               etype=m.etype)
    sub.young = None if m.young is None else np.ascontiguousarray(m.young[elems])
    sub.poisson = None if m.poisson is None else np.ascontiguousarray(m.poisson[elems])
    dof_eq, prescribed, _ = model.dof_map()
    g = (3 * nodes[:, None] + np.arange(3)[None, :]).reshape(-1)
    sub_free = dof_eq[g] >= 0
    spc_l = np.nonzero(~sub_free)[0]
    spc = (spc_l // 3, spc_l % 3, prescribed[g][spc_l])
    cl = None
    if model.cloads is not None:
        cn, cc, cv = (np.asarray(x) for x in model.cloads)
        keep = local[cn] >= 0
        cl = (local[cn[keep]], cc[keep], cv[keep])
    shard_model = Model(sub, model.materials, None if model.elem_mat is None else model.elem_mat[elems], spc, cl)
    eq_global = dof_eq[g][sub_free].astype(np.int64)
    # free equations are numbered in increasing global DOF order
    row0 = int((dof_eq[:3 * n0] >= 0).sum())
    n_rows = int((dof_eq[3 * n0:3 * n1] >= 0).sum())
    local_row0 = int(np.searchsorted(eq_global, row0))
    return Shard(rank, (n0, n1), shard_model, nodes, elems, eq_global, row0, n_rows, local_row0)


def owned_rows(shard: Shard, row_ptr, col_idx, vals, rhs=None):
    """The shard's owned rows in global numbering: (row_ptr from 0, global col_idx,
    vals, rhs) from the shard model's local CSR (numpy or torch arrays)."""
    rp = np.asarray(row_ptr)
    lo, hi = shard.local_row0, shard.local_row0 + shard.n_rows
    a, b = int(rp[lo]), int(rp[hi])
    out_rp = rp[lo:hi + 1] - a
    out_ci = shard.eq_global[np.asarray(col_idx)[a:b]]
    out_v = vals[a:b]
    out_r = None if rhs is None else rhs[lo:hi]
    return out_rp, out_ci, out_v, out_r


def owned_nodal(shard: Shard, local_vec):
    """Entries of the shard's owned nodes from a local nodal vector [3 * shard nodes]
    (f_int), in global node order."""
    n0, n1 = shard.node_range
    lo = int(np.searchsorted(shard.nodes, n0))
    return local_vec[3 * lo:3 * (lo + n1 - n0)]


def shard_state(shard: Shard, state, gauss_per_element: int):
    """Per-Gauss-point history of the shard's elements from the global [G, 13] array."""
    idx = (shard.elems[:, None] * gauss_per_element + np.arange(gauss_per_element)[None, :]).reshape(-1)
    return state[idx]


def owned_elements(shard: Shard):
    """Mask over the shard's elements: True where this rank owns the element's history,
    i.e. the element's first node is an owned node (every element has one owner)."""
    n0, n1 = shard.node_range
    first = shard.nodes[shard.model.mesh.conn[:, 0]]
    return (first >= n0) & (first < n1)
