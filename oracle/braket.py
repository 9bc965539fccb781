"""Double-layer (bra-ket) network for <psi|psi> (oracle; test infrastructure).

Restates ``src/braket.jl`` of CATN.jl for real FP64 tensors: ``braket_node``
(:75-195), ``cano_to!`` (:201-233, the same sweep as the MPSNode one),
``swap!`` (:510-562, which also swaps the layer tags), ``move!`` /
``move2tail!`` / ``move2head!`` (:570-611), ``eat!`` (:638-798, four cases),
``compress!`` / ``compress_opt!`` (:820-903, the MPSNode ones), the final
``braket_lognorm`` (:915-940) and ``contraction!`` (:960-1078).

One deliberate difference: the reference takes its edges in the iteration
order of a Julia Dict keyed by label (braket.jl:489-497), which is hash
order and cannot be reproduced outside Julia; here the edges are taken in
order of first appearance of their labels, scanning the tensors in order
and each tensor's labels in order.  In exact mode the value does not depend
on the order; the reference's own tests (test/test_braket.jl:246-347) check
exactly those order-free properties.
"""
import math

import numpy as np

from . import mps as M
from .linalg import tsvd
from .mps import rs

TRACE = None


class BraKetNode(M.MPSNode):
    """``BraKetNode`` (braket.jl:20-33): an MPSNode plus a ket/bra tag per site."""

    def __init__(self, mps, neighbor, layer, cano, chi, cutoff=1e-15, norm_method=1, svdopt=True, swapopt=True):
        super().__init__(mps, neighbor, cano, chi, cutoff, norm_method, svdopt, swapopt)
        self.layer = list(layer)


def _sweep(R, dleft, axes, chi, cutoff):
    """Left-to-right SVDs over ``axes`` of R (shape (dleft, *axes, rest...))."""
    sites = []
    for i in range(len(axes) - 1):
        Mx = rs(R, dleft * axes[i], R.size // (dleft * axes[i]))
        U, S, V, _ = tsvd(Mx, cutoff=cutoff, maxdim=chi, tag="braket_node")
        c = S.shape[0]
        sites.append(rs(U, dleft, axes[i], c))
        R = rs(S[:, None] * V.conj().T, c, R.size // (dleft * axes[i]))
        dleft = c
    return sites, R, dleft


def braket_node(Ti, ket_neighbors, phys_pos, chi=32, cutoff=1e-15, norm_method=1, svdopt=True, swapopt=False):
    """Ket sites then bra sites of E_i = sum_p T_i conj(T_i) (braket.jl:75-195)."""
    nd = Ti.ndim
    deg = nd - 1
    if deg < 1:
        raise ValueError("braket_node: degree-0 site (no virtual legs) is not supported.")
    if len(ket_neighbors) != deg:
        raise ValueError(f"braket_node: length(ket_neighbors)={len(ket_neighbors)}, expected {deg}")
    perm = [a for a in range(nd) if a != phys_pos - 1] + [phys_pos - 1]
    Tk = np.transpose(Ti, perm)
    dims = Tk.shape
    d = dims[deg]
    ket, R, dleft = _sweep(rs(Tk, 1, *dims), 1, list(dims[:deg]), chi, cutoff)
    ket.append(rs(R, dleft, dims[deg - 1], d))
    Tb = np.transpose(Tk.conj(), [deg] + list(range(deg)))
    bra, R, dleft = _sweep(Tb, d, list(dims[:deg]), chi, cutoff)
    bra.append(rs(R, dleft, dims[deg - 1], 1))
    node = BraKetNode(ket + bra, list(ket_neighbors) * 2, [True] * deg + [False] * deg, 1, chi, cutoff,
                      norm_method, svdopt, swapopt)
    M.left_canonical(node)
    return node


def find_leg(node, j, isket):
    """(braket.jl:287-292): 1-based site index of the (j, layer) leg, or 0."""
    for k in range(len(node.mps)):
        if node.neighbor[k] == j and node.layer[k] == isket:
            return k + 1
    return 0


def swap(node, i, j):
    """``swap!`` (braket.jl:510-562): the MPSNode swap, layer tags riding along."""
    err = M.swap(node, i, j)
    node.layer[i - 1], node.layer[j - 1] = node.layer[j - 1], node.layer[i - 1]
    return err


def move(node, a, b):
    err = 0.0
    step = 1 if b > a else -1
    for idx in range(a, b, step):
        err += swap(node, idx, idx + step)
    return err


class BraKetNetwork:
    """``BraKetNetwork`` (braket.jl:335-349)."""

    def __init__(self, tensors, edges, chi, cutoff, norm_method, svdopt, swapopt, loops=False):
        self.tensors = tensors
        self.loops = loops
        self.edges = edges          # list of (i, j), in processing order
        self.chi, self.cutoff, self.norm_method = chi, cutoff, norm_method
        self.svdopt, self.swapopt = svdopt, swapopt
        self.lnZ, self.psi = 0.0, 1.0
        self.maxdim_intermediate = 0


def braket_network(tensors, ixs, chi=64, cutoff=1e-15, norm_method=1, svdopt=True, swapopt=True, seed=1,
                   loops=False):
    """(braket.jl:369-508); edges in first-appearance order of their labels.
    ``loops=True`` restates the library's loopy extension (no reference
    counterpart): cycles are accepted, parallel bonds in the input are not."""
    n = len(tensors)
    if n != len(ixs):
        raise ValueError("braket_network: length(tensors) != length(ixs)")
    count, owners, order = {}, {}, []
    for i in range(n):
        for lbl in ixs[i]:
            if lbl not in count:
                order.append(lbl)
            count[lbl] = count.get(lbl, 0) + 1
            owners.setdefault(lbl, []).append(i + 1)
    for lbl, c in count.items():
        if c not in (1, 2):
            raise ValueError(f"braket_network: label {lbl} appears {c} times (expected 1 or 2)")
    for i in range(n):
        nphys = sum(1 for lbl in ixs[i] if count[lbl] == 1)
        if nphys != 1:
            raise ValueError(f"braket_network: tensor {i + 1} has {nphys} physical (open) labels, expected 1")
    parent = list(range(n + 1))

    def root(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    pairs = set()
    for lbl in order:
        if count[lbl] == 2 and loops:
            key = tuple(sorted(owners[lbl]))
            if key in pairs:
                raise ValueError(f"braket_network: tensors {key[0]} and {key[1]} share more than one label "
                                 "(parallel bonds are not supported)")
            pairs.add(key)
        elif count[lbl] == 2:
            a, b = root(owners[lbl][0]), root(owners[lbl][1])
            if a == b:
                raise ValueError("braket_network: virtual-bond graph contains a cycle — cyclic graphs are not "
                                 "supported in v1")
            parent[a] = b
    nodes = {}
    for i in range(n):
        phys, kn = 0, []
        for ax, lbl in enumerate(ixs[i]):
            if count[lbl] == 1:
                phys = ax + 1
            else:
                o = owners[lbl]
                kn.append(o[1] if o[0] == i + 1 else o[0])
        nodes[i + 1] = braket_node(np.asarray(tensors[i], dtype=np.float64), kn, phys, chi=chi, cutoff=cutoff,
                                   norm_method=norm_method, svdopt=svdopt, swapopt=swapopt)
    edges = [tuple(owners[lbl]) for lbl in order if count[lbl] == 2]
    return BraKetNetwork(nodes, edges, chi, cutoff, norm_method, svdopt, swapopt, loops)


def _norm(node, t):
    if node.norm_method == 1:
        return float(np.linalg.norm(t.reshape(-1)))
    if node.norm_method == 2:
        return float(np.max(np.abs(t)))
    return 1.0


def _finish(node, err):
    M.cano_to(node, len(node.mps))
    center = node.mps[node.cano - 1]
    nrm = _norm(node, center)
    if nrm <= node.cutoff:
        return 0.0, err, 1.0
    node.mps[-1] = node.mps[-1] / nrm
    return math.log(nrm), err, 1.0


def eat(ni, nj, j_id, i_id):
    """``eat!`` (braket.jl:638-798): contract the paired ket and bra legs."""
    err = 0.0
    n_i, n_j = len(ni.mps), len(nj.mps)
    bi = find_leg(ni, j_id, False)
    if bi == 0:
        raise ValueError(f"eat!: bra leg to neighbor {j_id} not found in node_i")
    err += move(ni, bi, n_i)
    ki = find_leg(ni, j_id, True)
    if ki == 0:
        raise ValueError(f"eat!: ket leg to neighbor {j_id} not found in node_i")
    err += move(ni, ki, n_i - 1)
    M.cano_to(ni, n_i)
    kj = find_leg(nj, i_id, True)
    if kj == 0:
        raise ValueError(f"eat!: ket leg to neighbor {i_id} not found in node_j")
    err += move(nj, kj, 1)
    bj = find_leg(nj, i_id, False)
    if bj == 0:
        raise ValueError(f"eat!: bra leg to neighbor {i_id} not found in node_j")
    err += move(nj, bj, 2)
    Aik, Aib, Ajk, Ajb = ni.mps[n_i - 2], ni.mps[n_i - 1], nj.mps[0], nj.mps[1]
    dl, Dk, Db, dr = Aik.shape[0], Aik.shape[1], Aib.shape[1], Ajb.shape[2]
    Wi = rs(np.einsum("ijk,kab->ijab", Aik, Aib), dl, Dk, Db)
    Wj = rs(np.einsum("ijk,kab->ijab", Ajk, Ajb), Dk, Db, dr)
    mat = np.einsum("iab,abj->ij", Wi, Wj)
    if n_i == 2 and n_j == 2:                     # case A
        z = float(np.sum(mat))
        ni.mps, ni.neighbor, ni.layer = [], [], []
        if abs(z) <= ni.cutoff:
            return 0.0, err, 1.0
        return math.log(abs(z)), err, z / abs(z)
    if n_i == 2:                                  # case B
        first = np.einsum("ijk,kab->iab", rs(mat, 1, 1, dr), nj.mps[2])
        ni.mps = [first] + nj.mps[3:]
        ni.neighbor = nj.neighbor[2:]
        ni.layer = nj.layer[2:]
        ni.cano = 1
        return _finish(ni, err)
    ni.mps[n_i - 3] = np.einsum("ijk,ka->ija", ni.mps[n_i - 3], mat)
    ni.cano = n_i - 2
    del ni.mps[-2:]
    del ni.neighbor[-2:]
    del ni.layer[-2:]
    if n_j > 2:                                   # case D (case C when n_j == 2)
        ni.mps.extend(nj.mps[2:])
        ni.neighbor.extend(nj.neighbor[2:])
        ni.layer.extend(nj.layer[2:])
    return _finish(ni, err)


def merge_leg(node, j, isket, cross):
    """Loopy extension: fuse the two legs of ``node`` pointing to ``j`` in one
    layer, as ``merge!`` (mps_node.jl:595-622) fuses a duplicate bond, the
    layer tags riding along with the swaps."""
    positions = [k + 1 for k in range(len(node.mps)) if node.neighbor[k] == j and node.layer[k] == isket]
    if len(positions) != 2:
        raise ValueError(f"merge: expected 2 legs to {j} in one layer, found {len(positions)}")
    idx1, idx2 = positions
    target = idx1 if cross else idx1 + 1
    err = move(node, idx2, target)
    del node.neighbor[target - 1]
    del node.layer[target - 1]
    M.cano_to(node, idx1)
    a, b = node.mps[idx1 - 1], node.mps[idx1]
    node.mps[idx1 - 1] = rs(np.einsum("ijk,kab->ijab", a, b), a.shape[0], a.shape[1] * b.shape[1], b.shape[2])
    del node.mps[idx1]
    M.cano_to(node, idx1)
    return err


def braket_lognorm(bk):
    """(braket.jl:915-940)"""
    total = 0.0
    for node in bk.tensors.values():
        if not node.mps:
            continue
        M.cano_to(node, len(node.mps))
        nrm = _norm(node, node.mps[node.cano - 1])
        if nrm <= node.cutoff:
            continue
        total += math.log(nrm)
    return total, 1.0


def contraction(bk):
    """``contraction!(bk) -> (lnZ, error, psi)`` (braket.jl:960-1078)."""
    err = 0.0
    bk.psi, bk.lnZ = 1.0, 0.0
    while bk.edges:
        i, j = bk.edges[0]
        ni, nj = bk.tensors[i], bk.tensors[j]
        if len(nj.mps) > len(ni.mps):
            i, j, ni, nj = j, i, nj, ni
        lnv, e, phase = eat(ni, nj, j, i)
        err += e
        bk.psi *= phase
        bk.lnZ += lnv
        err += M.compress_opt(ni) if bk.svdopt else M.compress(ni)
        for t in ni.mps:
            bk.maxdim_intermediate = max(bk.maxdim_intermediate, t.shape[1])
        bk.edges = [(a, b) for (a, b) in bk.edges if not ((a, b) == (i, j) or (a, b) == (j, i))]
        new, dups = [], []
        for (a, b) in bk.edges:
            if a == j or b == j:
                other = b if a == j else a
                on = bk.tensors[other]
                xk, yk = find_leg(on, i, True), find_leg(on, j, True)
                xb, yb = find_leg(on, i, False), find_leg(on, j, False)
                on.neighbor = [i if v == j else v for v in on.neighbor]
                if xk > 0:   # a second doubled bond between i and other (loops only)
                    dups.append((other, xk > yk, xb > yb))
                    continue
                new.append((i, other) if a == j else (other, i))
            else:
                new.append((a, b))
        bk.edges = new
        if dups and not bk.loops:
            raise ValueError("contraction!: parallel doubled bonds in a network built without loops")
        for (k, ck, cb) in dups:
            nk = bk.tensors[k]
            err += merge_leg(nk, i, True, ck)
            err += merge_leg(nk, i, False, cb)
            err += merge_leg(ni, k, True, False)
            err += merge_leg(ni, k, False, False)
            for t in nk.mps:
                bk.maxdim_intermediate = max(bk.maxdim_intermediate, t.shape[1])
        if dups:
            err += M.compress_opt(ni) if bk.svdopt else M.compress(ni)
            for t in ni.mps:
                bk.maxdim_intermediate = max(bk.maxdim_intermediate, t.shape[1])
        if TRACE is not None:
            TRACE.append((i, j, tuple(M.shape(ni)), tuple(int(x) for x in ni.layer)))
        del bk.tensors[j]
    ln, sg = braket_lognorm(bk)
    bk.lnZ += ln
    bk.psi *= sg
    return bk.lnZ, err, bk.psi


def exact_norm(tensors, ixs):
    """<psi|psi> by dense contraction (test/test_braket.jl exact_norm)."""
    from .exact import exact_contract
    ket = exact_contract([np.asarray(t) for t in tensors], ixs)
    return float(np.sum(ket * np.conj(ket)))
