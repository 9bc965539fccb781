"""Network engine: graph bookkeeping, edge selection, bond cutting and the
``contraction!`` loop (oracle; test infrastructure).

Restates ``src/tensor_network.jl`` of CATN.jl.  ``TRACE`` (when a list) records
one tuple per contraction step -- the integer trace that the CUDA library must
reproduce bit for bit:

    (i, j, reversed_i, reversed_j, duplicates, phys_dims_of_i_after_step)
"""
import math

import numpy as np

from . import mps as M
from .linalg import tsvd, thin_qr

TRACE = None


def _round_half_even(x):
    """Julia ``round(Int, x)`` (ties to even)."""
    return int(round(x))  # Python's round() is round-half-even


class TensorNetwork:
    """``TensorNetwork{T,AT}`` (tensor_network.jl:1-22)."""

    def __init__(self, tensors, Dmax=32, chi=32, cutoff=1e-15, norm_method=1, select=1,
                 reverse=True, svdopt=True, swapopt=True, compress=False, cut_bond=False,
                 seed=1, n=None, beta=1.0, num_isolated=0):
        self.tensors = tensors          # dict: node id (1-based) -> MPSNode
        self.Dmax = int(Dmax)
        self.chi = int(chi)
        self.cutoff = float(cutoff)
        self.norm_method = int(norm_method)
        self.select = int(select)
        self.reverse = bool(reverse)
        self.svdopt = bool(svdopt)
        self.swapopt = bool(swapopt)
        self.compress = bool(compress)
        self.cut_bond = bool(cut_bond)
        self.edge_count = {}
        self.lnZ = 0.0
        self.sign = 1.0
        self.psi = 1.0
        self.maxdim_intermediate = -1
        self.num_isolated = num_isolated
        self.seed = seed
        self.n = len(tensors) if n is None else n
        self.beta = float(beta)

    @classmethod
    def from_tensors(cls, tensors, ixs, Dmax=32, chi=32, cutoff=1e-15, norm_method=1,
                     select=1, reverse=True, svdopt=True, swapopt=True, compress=False,
                     cut_bond=False, seed=1):
        """Label-graph constructor (tensor_network.jl:41-140)."""
        n = len(tensors)
        assert len(ixs) == n, "tensors and ixs must have the same length"
        for t in range(n):
            seen = set()
            for lbl in ixs[t]:
                if lbl in seen:
                    raise ValueError(f"Self-loop detected: label {lbl} appears twice in tensor {t + 1}'s index list")
                seen.add(lbl)
        label_map = {}
        for t in range(n):
            for k, lbl in enumerate(ixs[t]):
                label_map.setdefault(lbl, []).append((t + 1, k + 1))
        for lbl, occ in label_map.items():
            if len(occ) > 2:
                raise ValueError(f"Label {lbl} appears in {len(occ)} tensors (max 2 allowed)")
        sentinel = 0
        neighbor_vecs = [[0] * len(ixs[t]) for t in range(n)]
        # Julia iterates a Dict here; sentinel numbering only needs uniqueness.
        for lbl, occ in label_map.items():
            if len(occ) == 2:
                (t1, k1), (t2, k2) = occ
                neighbor_vecs[t1 - 1][k1 - 1] = t2
                neighbor_vecs[t2 - 1][k2 - 1] = t1
            else:
                sentinel -= 1
                t, k = occ[0]
                neighbor_vecs[t - 1][k - 1] = sentinel
        nodes = {}
        for t in range(n):
            nodes[t + 1] = M.MPSNode.from_tensor(tensors[t], neighbor_vecs[t], chi=chi, cutoff=cutoff,
                                                 norm_method=norm_method, svdopt=svdopt,
                                                 swapopt=swapopt)
        num_isolated = sum(1 for t in range(n) if all(nb < 0 for nb in neighbor_vecs[t]))
        return cls(nodes, Dmax=Dmax, chi=chi, cutoff=cutoff, norm_method=norm_method,
                   select=select, reverse=reverse, svdopt=svdopt, swapopt=swapopt,
                   compress=compress, cut_bond=cut_bond, seed=seed, n=n,
                   num_isolated=num_isolated)


# ---------------------------------------------------------------------------
# edge-cost bookkeeping (tensor_network.jl:152-236)
# ---------------------------------------------------------------------------

def dim_after_merge(tn, i, j):
    """``round(Int, logdim(i) + logdim(j) - 2 logdim(i, idx_j_in_i))`` (:152-155)."""
    ni = tn.tensors[i]
    idx = M.find_neighbor(ni, j)
    return _round_half_even(M.logdim(ni) + M.logdim(tn.tensors[j]) - 2 * M.logdim(ni, idx))


def count_add_edges(tn, edges):
    """Append each pair to its cost bucket (:167-176)."""
    for i, j in edges:
        cost = dim_after_merge(tn, i, j)
        tn.edge_count.setdefault(cost, []).append((i, j))


def count_add_nodes(tn, nodes):
    """Collect incident real bonds, dedupe, sort lexicographically, add (:185-197)."""
    edges = set()
    for i in nodes:
        if i <= 0:
            continue
        for j in tn.tensors[i].neighbor:
            if j <= 0:
                continue
            edges.add((min(i, j), max(i, j)))
    count_add_edges(tn, sorted(edges))


def count_remove_nodes(tn, nodes):
    """Remove incident bonds from the bucket of their *current* cost (:213-225)."""
    for node_id in nodes:
        if node_id <= 0:
            continue
        for nb in tn.tensors[node_id].neighbor:
            if nb <= 0:
                continue
            i, j = min(node_id, nb), max(node_id, nb)
            cost = dim_after_merge(tn, i, j)
            if cost in tn.edge_count:
                tn.edge_count[cost] = [p for p in tn.edge_count[cost] if p != (i, j)]


def select_edge_init(tn):
    """(:233-236)"""
    tn.edge_count = {}
    count_add_nodes(tn, list(tn.tensors.keys()))


def select_edge_min_dim(tn):
    """Cheapest non-empty bucket, first pair (:248-253)."""
    cost = min(k for k, v in tn.edge_count.items() if v)
    tn.maxdim_intermediate = max(tn.maxdim_intermediate, cost)
    return tn.edge_count[cost][0]


def select_edge_min_dim_triangle(tn):
    """Cheapest bucket, pair with most common neighbours, first max wins (:262-288)."""
    cost = min(k for k, v in tn.edge_count.items() if v)
    tn.maxdim_intermediate = max(tn.maxdim_intermediate, cost)
    cands = tn.edge_count[cost]
    best_pair, best_count = cands[0], -1
    for (i, j) in cands:
        neigh_j = {nb for nb in tn.tensors[j].neighbor if nb > 0 and nb != i}
        both = sum(1 for k in neigh_j if M.find_neighbor(tn.tensors[k], i) > 0)
        if both > best_count:
            best_count, best_pair = both, (i, j)
    return best_pair


def select_edge_sequentially(tn):
    """Edge minimising ``i+j`` (:300-316).

    The reference scans ``keys(tn.tensors)`` (Julia Dict order, hash-defined);
    this restatement scans node ids in ascending order, so ties in ``i+j`` are
    broken by the smaller ``i``.
    """
    best, bestsum = None, None
    for i in sorted(tn.tensors.keys()):
        for nb in tn.tensors[i].neighbor:
            if nb <= 0 or not i < nb:
                continue
            s = i + nb
            if bestsum is None or s < bestsum:
                bestsum, best = s, (i, nb)
    if best is None:
        raise ValueError("select_edge_sequentially: no edges remain")
    return best


# ---------------------------------------------------------------------------
# physical-bond truncation (tensor_network.jl:342-477)
# ---------------------------------------------------------------------------

def _bond_ends(tn, i, idx_j_in_i, name):
    node_i = tn.tensors[i]
    j = node_i.neighbor[idx_j_in_i - 1]
    if j <= 0:
        raise ValueError(f"{name}: leg {idx_j_in_i} of node {i} is an open leg (no neighbor)")
    node_j = tn.tensors[j]
    idx_i_in_j = M.find_neighbor(node_j, i)
    if idx_i_in_j == 0:
        raise ValueError(f"{name}: node {i} not found as neighbor of node {j}")
    return node_i, node_j, idx_i_in_j


def _split_store(tn, node_i, node_j, idx_j_in_i, idx_i_in_j, U, S, V, disc, Ai_shape, Aj_shape,
                 qi=None, qj=None):
    myd = max(1, min(S.shape[0], tn.Dmax))
    extra = float(np.sum(S[myd:])) if myd < S.shape[0] else 0.0
    err = disc + extra
    S, U, V = S[:myd], U[:, :myd], V[:, :myd]
    sq = np.sqrt(S)
    mati = U * sq[None, :]
    matj = V.conj() * sq[None, :]
    if qi is not None:
        mati = qi @ mati
    if qj is not None:
        matj = qj @ matj
    da_l, _, da_r = Ai_shape
    db_l, _, db_r = Aj_shape
    node_i.mps[idx_j_in_i - 1] = np.transpose(M.rs(mati, da_l, da_r, myd), (0, 2, 1))
    node_j.mps[idx_i_in_j - 1] = np.transpose(M.rs(matj, db_l, db_r, myd), (0, 2, 1))
    return err, myd


def cut_bondim(tn, i, idx_j_in_i):
    """Plain bond cut without QR or canonicalisation (:342-388)."""
    if tn.Dmax < 0:
        return 0.0
    node_i, node_j, idx_i_in_j = _bond_ends(tn, i, idx_j_in_i, "cut_bondim!")
    Ai, Aj = node_i.mps[idx_j_in_i - 1], node_j.mps[idx_i_in_j - 1]
    da_l, d, da_r = Ai.shape
    db_l, _, db_r = Aj.shape
    mati = M.rs(np.transpose(Ai, (0, 2, 1)), da_l * da_r, d)
    matj = M.rs(np.transpose(Aj, (0, 2, 1)), db_l * db_r, d)
    U, S, V, disc = tsvd(mati @ matj.T, cutoff=tn.cutoff, tag="cut")
    err, _ = _split_store(tn, node_i, node_j, idx_j_in_i, idx_i_in_j, U, S, V, disc,
                          Ai.shape, Aj.shape)
    return err


def cut_bondim_opt(tn, i, idx_j_in_i):
    """Bond cut with canonicalisation and QR pre-reduction (:399-477)."""
    if tn.Dmax < 0:
        return 0.0
    node_i, node_j, idx_i_in_j = _bond_ends(tn, i, idx_j_in_i, "cut_bondim_opt!")
    M.cano_to(node_i, idx_j_in_i)
    M.cano_to(node_j, idx_i_in_j)
    Ai, Aj = node_i.mps[idx_j_in_i - 1], node_j.mps[idx_i_in_j - 1]
    da_l, d, da_r = Ai.shape
    db_l, _, db_r = Aj.shape
    mati = M.rs(np.transpose(Ai, (0, 2, 1)), da_l * da_r, d)
    matj = M.rs(np.transpose(Aj, (0, 2, 1)), db_l * db_r, d)
    qi = qj = None
    if mati.shape[0] > mati.shape[1]:
        qi, ri = thin_qr(mati)
    else:
        ri = mati
    if matj.shape[0] > matj.shape[1]:
        qj, rj = thin_qr(matj)
    else:
        rj = matj
    U, S, V, disc = tsvd(ri @ rj.T, cutoff=tn.cutoff, tag="cut_opt")
    err, myd = _split_store(tn, node_i, node_j, idx_j_in_i, idx_i_in_j, U, S, V, disc,
                            Ai.shape, Aj.shape, qi, qj)
    M._log("cut", da_l * da_r, db_l * db_r, d, 0, myd)
    return err


# ---------------------------------------------------------------------------
# lognorm fold, result tensor, main loop (tensor_network.jl:489-717)
# ---------------------------------------------------------------------------

def network_lognorm(tn):
    """(:489-501)"""
    total, sign = 0.0, 1.0
    for node in tn.tensors.values():
        if not all(s.shape[1] == 1 for s in node.mps):
            continue
        ln, sg = M.lognorm(node)
        total += ln
        sign = sign * sg
    return total, sign


def result_tensor(tn):
    """(:517-523)"""
    open_nodes = [nd for nd in tn.tensors.values() if not all(s.shape[1] == 1 for s in nd.mps)]
    if not open_nodes:
        return np.ones(())
    if len(open_nodes) != 1:
        raise ValueError(f"result_tensor: expected one surviving open-leg node, got {len(open_nodes)}")
    return M.mps2raw(open_nodes[0])


def has_real_edges(tn):
    """(:535-542)"""
    return any(nb > 0 for node in tn.tensors.values() for nb in node.neighbor)


def contraction(tn):
    """``contraction!(tn) -> (lnZ, error, psi)`` (tensor_network.jl:556-717)."""
    error = 0.0
    tn.psi = 1.0
    tn.lnZ = 0.0
    if tn.select in (0, 1) and not tn.edge_count:
        select_edge_init(tn)
    while has_real_edges(tn):
        if tn.select == 0:
            i, j = select_edge_min_dim(tn)
        elif tn.select == 1:
            i, j = select_edge_min_dim_triangle(tn)
        else:
            i, j = select_edge_sequentially(tn)
        node_i, node_j = tn.tensors[i], tn.tensors[j]
        if M.order(node_j) > M.order(node_i):
            i, j = j, i
            node_i, node_j = node_j, node_i
        affected = [i, j] + list(node_i.neighbor) + list(node_j.neighbor)
        if tn.select in (0, 1):
            count_remove_nodes(tn, affected)
        neigh_j = list(node_j.neighbor)
        idx_j_in_i = M.find_neighbor(node_i, j)
        idx_i_in_j = M.find_neighbor(node_j, i)
        rev_i = rev_j = False
        if tn.reverse:
            if idx_j_in_i < -(-len(node_i.neighbor) // 2):
                M.reverse(node_i)
                idx_j_in_i = M.find_neighbor(node_i, j)
                rev_i = True
            if idx_i_in_j >= -(-len(node_j.neighbor) // 2):
                M.reverse(node_j)
                neigh_j = list(node_j.neighbor)
                idx_i_in_j = M.find_neighbor(node_j, i)
                rev_j = True
        duplicate = []
        for l in range(1, len(neigh_j) + 1):
            if l == idx_i_in_j:
                continue
            k = neigh_j[l - 1]
            if k <= 0:
                continue
            idx_k_in_i = M.find_neighbor(node_i, k)
            node_k = tn.tensors[k]
            idx_i_in_k = M.find_neighbor(node_k, i)
            idx_j_in_k = M.delete_neighbor(node_k, j)
            M.add_neighbor(node_k, i, idx_j_in_k)
            if idx_k_in_i > 0:
                duplicate.append(k)
                cross = idx_i_in_k > idx_j_in_k
                error += M.merge(node_k, i, cross=cross)
        lnv, err, phase = M.eat(node_i, node_j, idx_j_in_i, idx_i_in_j)
        error += err
        tn.psi = tn.psi * phase
        tn.lnZ += lnv
        for k in duplicate:
            M.merge(node_i, k, cross=False)
            idx_k_in_i = M.find_neighbor(node_i, k)
            if tn.cut_bond or (tn.Dmax > 0 and node_i.mps[idx_k_in_i - 1].shape[1] > tn.Dmax):
                error += cut_bondim_opt(tn, i, idx_k_in_i)
        M.clear(node_j)
        if tn.compress:
            if tn.svdopt:
                M.compress_opt(node_i)
            else:
                M.compress(node_i)
        if tn.select in (0, 1):
            count_add_nodes(tn, [i] + list(node_i.neighbor))
        for t in node_i.mps:
            if t.shape[1] > tn.maxdim_intermediate:
                tn.maxdim_intermediate = t.shape[1]
        if TRACE is not None:
            TRACE.append((i, j, rev_i, rev_j, tuple(duplicate), tuple(M.shape(node_i))))
    ln, sg = network_lognorm(tn)
    tn.sign = sg
    tn.lnZ += ln
    return tn.lnZ, error, tn.psi
