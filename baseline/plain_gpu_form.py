"""The plain GPU form of CATN's ``contraction!``: a PyTorch FP64 restatement
that issues one library call per tensor operation (``torch.einsum``,
``torch.linalg.svd``, ``torch.linalg.qr``) from a host loop.

This is the analogue of running the reference on a GPU through
``adapt(CuArray, tn)`` (``src/adapt.jl:6-24``): every site tensor lives on the
device, every rank decision (``count(S .> cutoff)``) and every norm is read
back to the host before the next call, and instances run one after another.
It is a measured comparison line for the batched engine, not part of the
library, and it runs no code of the library.

Follows ``src/linalg_utils.jl:15-58``, ``src/mps_node.jl:72-622``,
``src/tensor_network.jl:152-717`` and ``src/ising.jl:20-227``.  Sites are
``(left, phys, right)`` tensors with column-major reshapes, positions are
1-based, as in the reference.
"""
import math

import torch


def rs(a, *shape):
    """Column-major reshape (Julia ``reshape``)."""
    nd = a.dim()
    b = a.permute(*range(nd - 1, -1, -1)) if nd > 1 else a
    b = b.reshape(*shape[::-1])
    return b.permute(*range(len(shape) - 1, -1, -1)) if len(shape) > 1 else b


def flat(a):
    """Column-major flatten (Julia ``vec``)."""
    return a.permute(*range(a.dim() - 1, -1, -1)).reshape(-1)


# ---------------------------------------------------------------------------
# linalg_utils.jl
# ---------------------------------------------------------------------------

def tsvd(A, cutoff, maxdim=None):
    """``tsvd`` (linalg_utils.jl:15-28): thin SVD, keep ``count(S > cutoff)``
    (at least one, at most ``maxdim``), return the discarded sum of values."""
    U, S, Vh = torch.linalg.svd(A, full_matrices=False)
    nfull = S.shape[0]
    nkeep = int((S > cutoff).sum().item())
    nkeep = 1 if nkeep == 0 else min(nkeep, nfull if maxdim is None else maxdim)
    disc = float(S[nkeep:].sum().item()) if nkeep < nfull else 0.0
    return U[:, :nkeep], S[:nkeep], Vh[:nkeep, :].mH, disc


def rsvd(A, k, oversample=10, power=10, gen=None):
    """``rsvd`` (linalg_utils.jl:44-58) with a seeded sketch."""
    n = A.shape[1]
    p = min(n, oversample * k)
    G = torch.randn(n, p, dtype=A.dtype, device=A.device, generator=gen)
    Y = A @ G
    for _ in range(power):
        Y, _ = torch.linalg.qr(A @ (A.mH @ Y))
    Q, _ = torch.linalg.qr(Y)
    Ub, S, Vh = torch.linalg.svd(Q.mH @ A, full_matrices=False)
    kk = min(k, Ub.shape[1])
    return (Q @ Ub)[:, :kk], S[:kk], Vh[:kk, :].mH


# ---------------------------------------------------------------------------
# mps_node.jl
# ---------------------------------------------------------------------------

class Node:
    """``MPSNode`` (mps_node.jl:1-29): site list, neighbour ids, centre."""

    __slots__ = ("mps", "neighbor", "cano")

    def __init__(self):
        self.mps, self.neighbor, self.cano = [], [], 0


class Params:
    def __init__(self, Dmax=32, chi=32, cutoff=1e-15, norm_method=1, select=1, reverse=True,
                 svdopt=True, swapopt=True, compress=False, cut_bond=False):
        self.Dmax, self.chi, self.cutoff = int(Dmax), int(chi), float(cutoff)
        self.norm_method, self.select, self.reverse = int(norm_method), int(select), bool(reverse)
        self.svdopt, self.swapopt = bool(svdopt), bool(swapopt)
        self.compress, self.cut_bond = bool(compress), bool(cut_bond)


def cano_to(P, node, idx):
    """``cano_to!`` (mps_node.jl:72-104)."""
    if idx == 0:
        idx = len(node.mps)
    if node.cano == idx:
        return
    if node.cano < idx:
        for i in range(node.cano, idx):
            t = node.mps[i - 1]
            dl, d, dr = t.shape
            U, S, V, _ = tsvd(rs(t, dl * d, dr), 0.0)
            nkeep = int((S > P.cutoff).sum().item()) or S.shape[0]
            node.mps[i - 1] = rs(U[:, :nkeep], dl, d, nkeep)
            R = S[:nkeep, None] * V[:, :nkeep].mH
            node.mps[i] = torch.einsum("ij,jab->iab", R, node.mps[i])
            node.cano = i + 1
    else:
        for i in range(node.cano, idx, -1):
            t = node.mps[i - 1]
            dl, d, dr = t.shape
            U, S, V, _ = tsvd(rs(t.permute(1, 2, 0), d * dr, dl), 0.0)
            nkeep = int((S > P.cutoff).sum().item()) or S.shape[0]
            node.mps[i - 1] = rs(U[:, :nkeep], d, dr, nkeep).permute(2, 0, 1)
            R = S[:nkeep, None] * V[:, :nkeep].mH
            node.mps[i - 2] = torch.einsum("abc,cd->abd", node.mps[i - 2], R.T)
            node.cano = i - 1


def swap(P, node, i, j, gen=None):
    """``swap!`` (mps_node.jl:126-178); returns the discarded sum."""
    mps = node.mps
    if node.cano != i and node.cano != j:
        cano_to(P, node, i if abs(node.cano - i) < abs(node.cano - j) else j)
    tl, tr = (mps[i - 1], mps[j - 1]) if i < j else (mps[j - 1], mps[i - 1])
    d0, d1, d2, d3 = tl.shape[0], tr.shape[1], tl.shape[1], tr.shape[2]
    Mx = rs(torch.einsum("ijk,kab->iajb", tl, tr), d0 * d1, d2 * d3)
    rows, cols = Mx.shape
    if P.swapopt and ((rows > 7000 and cols > 7000) or rows > 20000 or cols > 20000):
        U, S, V = rsvd(Mx, P.chi, gen=gen)
        err = 0.0
    else:
        U, S, V, err = tsvd(Mx, P.cutoff, P.chi)
    myd = S.shape[0]
    if i < j:
        mps[i - 1] = rs(U, d0, d1, myd)
        mps[j - 1] = rs(S[:, None] * V.mH, myd, d2, d3)
    else:
        mps[j - 1] = rs(U * S[None, :], d0, d1, myd)
        mps[i - 1] = rs(V.mH, myd, d2, d3)
    node.cano = j
    nb = node.neighbor
    nb[i - 1], nb[j - 1] = nb[j - 1], nb[i - 1]
    return err


def move(P, node, a, b):
    """``move!`` (mps_node.jl:186-199)."""
    err = 0.0
    step = 1 if b > a else -1
    for idx in range(a, b, step):
        err += swap(P, node, idx, idx + step)
    return err


def move2tail(P, node, idx):
    """``move2tail!`` (mps_node.jl:208-217)."""
    err = move(P, node, idx, len(node.mps))
    cano_to(P, node, len(node.mps))
    return err


def move2head(P, node, idx):
    """``move2head!`` (mps_node.jl:225-229)."""
    err = move(P, node, idx, 1)
    cano_to(P, node, 1)
    return err


def reverse(node):
    """``reverse!`` (mps_node.jl:238-244)."""
    if len(node.mps) <= 1:
        return
    node.mps = [t.permute(2, 1, 0) for t in node.mps[::-1]]
    node.neighbor.reverse()
    node.cano = len(node.mps) + 1 - node.cano


def find_neighbor(node, j):
    """(mps_node.jl:257-260): 1-based position or 0."""
    try:
        return node.neighbor.index(j) + 1
    except ValueError:
        return 0


def logdim(node, idx=None):
    """(mps_node.jl:299-311): log2 of the phys dims, a left fold over sites."""
    if idx is not None:
        return math.log2(float(node.mps[idx - 1].shape[1]))
    s = 0.0
    for k, t in enumerate(node.mps):
        v = math.log2(float(t.shape[1]))
        s = v if k == 0 else s + v
    return s


def _norm(P, t):
    if P.norm_method == 1:
        return float(torch.linalg.vector_norm(t).item())
    if P.norm_method == 2:
        return float(t.abs().max().item())
    return 1.0


def compress_opt(P, node):
    """``compress_opt!`` (mps_node.jl:394-447)."""
    err = 0.0
    if not node.mps:
        return err
    node.cano = 1
    cano_to(P, node, len(node.mps))
    mps = node.mps
    for j in range(len(mps), 1, -1):
        i = j - 1
        tl, tr = mps[i - 1], mps[j - 1]
        d0, d1, d2, d3, dd = tl.shape[0], tl.shape[1], tr.shape[1], tr.shape[2], tl.shape[2]
        matl, matr = rs(tl, d0 * d1, dd), rs(tr, dd, d2 * d3)
        fl, fr = matl.shape[0] > matl.shape[1], matr.shape[0] < matr.shape[1]
        Ql, Rl = torch.linalg.qr(matl) if fl else (None, matl)
        Qr, Rr = torch.linalg.qr(matr.mH) if fr else (None, matr.mH)
        U, S, V, e = tsvd(Rl @ Rr.mH, P.cutoff, P.chi)
        err += e
        myd = S.shape[0]
        U = U * S[None, :]
        if fl:
            U = Ql @ U
        if fr:
            V = Qr @ V
        mps[i - 1] = rs(U, d0, d1, myd)
        mps[j - 1] = rs(V.mH, myd, d2, d3)
    node.cano = 1
    return err


def compress(P, node):
    """``compress!`` (mps_node.jl:356-376)."""
    err = 0.0
    if not node.mps:
        return err
    node.cano = 1
    cano_to(P, node, len(node.mps))
    mps = node.mps
    for j in range(len(mps), 1, -1):
        i = j - 1
        tl, tr = mps[i - 1], mps[j - 1]
        d0, d1, d2, d3 = tl.shape[0], tl.shape[1], tr.shape[1], tr.shape[2]
        U, S, V, e = tsvd(rs(torch.einsum("ijk,kab->ijab", tl, tr), d0 * d1, d2 * d3), P.cutoff, P.chi)
        err += e
        myd = S.shape[0]
        mps[i - 1] = rs(U * S[None, :], d0, d1, myd)
        mps[j - 1] = rs(V.mH, myd, d2, d3)
    node.cano = 1
    return err


def eat(P, node, nodej, idx, idxi):
    """``eat!`` (mps_node.jl:463-575); returns (lognorm, error, phase)."""
    err = 0.0
    if len(node.mps) == 1:                      # (a) both leaves
        r = float((flat(node.mps[0]) * flat(nodej.mps[0])).sum().item())
        node.mps.clear()
        del node.neighbor[idx - 1]
        if abs(r) <= P.cutoff:
            return 0.0, 0.0, 1.0
        return math.log(abs(r)), 0.0, r / abs(r)
    err += move2tail(P, node, idx)
    last = node.mps[-1]
    mati = rs(last, last.shape[0], last.shape[1])
    if len(nodej.mps) == 1:                     # (b) nodej is a leaf
        tj = nodej.mps[0]
        new = torch.einsum("ijk,ka->ija", node.mps[-2], mati @ rs(tj, tj.shape[1], 1))
        nrm = _norm(P, new)
        node.mps[-2] = new
        node.cano -= 1
        node.mps.pop()
        node.neighbor.pop()
        if nrm <= P.cutoff:
            return 0.0, err, 1.0
        node.mps[-1] = node.mps[-1] / nrm
        return math.log(nrm), err, 1.0
    err += move2head(P, nodej, idxi)            # (c) general
    h = nodej.mps[0]
    node.mps[-2] = torch.einsum("ijk,ka->ija", node.mps[-2], mati @ rs(h, h.shape[1], h.shape[2]))
    node.mps.pop()
    node.cano = len(node.mps)
    node.mps.extend(nodej.mps[1:])
    node.neighbor.pop()
    node.neighbor.extend(nodej.neighbor[1:])
    cano_to(P, node, len(node.mps))
    center = node.mps[node.cano - 1]
    nrm = _norm(P, center)
    if nrm <= P.cutoff:
        return 0.0, err, 1.0
    node.mps[node.cano - 1] = center / nrm
    return math.log(nrm), err, 1.0


def merge(P, node, j, cross=False):
    """``merge!`` (mps_node.jl:595-622)."""
    pos = [k + 1 for k, v in enumerate(node.neighbor) if v == j]
    if len(pos) != 2:
        raise ValueError(f"merge!: expected exactly 2 sites with neighbor {j}, found {len(pos)}")
    idx1, idx2 = pos
    target = idx1 if cross else idx1 + 1
    err = move(P, node, idx2, target)
    del node.neighbor[target - 1]
    cano_to(P, node, idx1)
    a, b = node.mps[idx1 - 1], node.mps[idx1]
    node.mps[idx1 - 1] = rs(torch.einsum("ijk,kab->ijab", a, b), a.shape[0], a.shape[1] * b.shape[1], b.shape[2])
    del node.mps[idx1]
    cano_to(P, node, idx1)
    return err


# ---------------------------------------------------------------------------
# tensor_network.jl
# ---------------------------------------------------------------------------

class Network:
    """``TensorNetwork`` (tensor_network.jl:1-22) restricted to what
    ``contraction!`` reads."""

    def __init__(self, nodes, P, n, beta):
        self.t, self.P, self.n, self.beta = nodes, P, n, beta
        self.edge_count = {}
        self.maxdim = -1


def dim_after_merge(tn, i, j):
    """(tensor_network.jl:152-155), Julia ``round`` ties to even."""
    ni = tn.t[i]
    return int(round(logdim(ni) + logdim(tn.t[j]) - 2 * logdim(ni, find_neighbor(ni, j))))


def count_add_nodes(tn, nodes):
    """(tensor_network.jl:167-197)."""
    edges = set()
    for i in nodes:
        if i > 0:
            edges.update((min(i, j), max(i, j)) for j in tn.t[i].neighbor if j > 0)
    for i, j in sorted(edges):
        tn.edge_count.setdefault(dim_after_merge(tn, i, j), []).append((i, j))


def count_remove_nodes(tn, nodes):
    """(tensor_network.jl:213-225)."""
    for a in nodes:
        if a <= 0:
            continue
        for b in tn.t[a].neighbor:
            if b <= 0:
                continue
            i, j = min(a, b), max(a, b)
            c = dim_after_merge(tn, i, j)
            if c in tn.edge_count:
                tn.edge_count[c] = [p for p in tn.edge_count[c] if p != (i, j)]


def select_edge(tn):
    """``select_edge_min_dim`` / ``_triangle`` / ``_sequentially``
    (tensor_network.jl:248-316); ties in ``select=2`` go to the smaller id."""
    if tn.P.select == 2:
        best, bs = None, None
        for i in sorted(tn.t):
            for nb in tn.t[i].neighbor:
                if nb > i and (bs is None or i + nb < bs):
                    bs, best = i + nb, (i, nb)
        return best
    cost = min(k for k, v in tn.edge_count.items() if v)
    tn.maxdim = max(tn.maxdim, cost)
    cands = tn.edge_count[cost]
    if tn.P.select == 0:
        return cands[0]
    best, bc = cands[0], -1
    for (i, j) in cands:
        nj = {nb for nb in tn.t[j].neighbor if nb > 0 and nb != i}
        c = sum(1 for k in nj if find_neighbor(tn.t[k], i) > 0)
        if c > bc:
            bc, best = c, (i, j)
    return best


def cut_bondim_opt(tn, i, idx_j_in_i):
    """``cut_bondim_opt!`` (tensor_network.jl:399-477)."""
    P = tn.P
    ni = tn.t[i]
    j = ni.neighbor[idx_j_in_i - 1]
    nj = tn.t[j]
    idx_i_in_j = find_neighbor(nj, i)
    cano_to(P, ni, idx_j_in_i)
    cano_to(P, nj, idx_i_in_j)
    Ai, Aj = ni.mps[idx_j_in_i - 1], nj.mps[idx_i_in_j - 1]
    al, d, ar = Ai.shape
    bl, _, br = Aj.shape
    mati, matj = rs(Ai.permute(0, 2, 1), al * ar, d), rs(Aj.permute(0, 2, 1), bl * br, d)
    qi, ri = torch.linalg.qr(mati) if mati.shape[0] > mati.shape[1] else (None, mati)
    qj, rj = torch.linalg.qr(matj) if matj.shape[0] > matj.shape[1] else (None, matj)
    U, S, V, disc = tsvd(ri @ rj.T, P.cutoff)
    myd = max(1, min(S.shape[0], P.Dmax))
    err = disc + (float(S[myd:].sum().item()) if myd < S.shape[0] else 0.0)
    sq = torch.sqrt(S[:myd])
    mi, mj = U[:, :myd] * sq[None, :], V[:, :myd].conj() * sq[None, :]
    if qi is not None:
        mi = qi @ mi
    if qj is not None:
        mj = qj @ mj
    ni.mps[idx_j_in_i - 1] = rs(mi, al, ar, myd).permute(0, 2, 1)
    nj.mps[idx_i_in_j - 1] = rs(mj, bl, br, myd).permute(0, 2, 1)
    return err


def contraction(tn, gen=None):
    """``contraction!(tn) -> (lnZ, error, psi)`` (tensor_network.jl:556-717)."""
    P, T = tn.P, tn.t
    error, psi, lnZ = 0.0, 1.0, 0.0
    if P.select in (0, 1):
        tn.edge_count = {}
        count_add_nodes(tn, list(T))
    while any(nb > 0 for nd in T.values() for nb in nd.neighbor):
        i, j = select_edge(tn)
        ni, nj = T[i], T[j]
        if len(nj.mps) > len(ni.mps):
            i, j, ni, nj = j, i, nj, ni
        if P.select in (0, 1):
            count_remove_nodes(tn, [i, j] + ni.neighbor + nj.neighbor)
        neigh_j = list(nj.neighbor)
        idx_j_in_i, idx_i_in_j = find_neighbor(ni, j), find_neighbor(nj, i)
        if P.reverse:
            if idx_j_in_i < -(-len(ni.neighbor) // 2):
                reverse(ni)
                idx_j_in_i = find_neighbor(ni, j)
            if idx_i_in_j >= -(-len(nj.neighbor) // 2):
                reverse(nj)
                neigh_j = list(nj.neighbor)
                idx_i_in_j = find_neighbor(nj, i)
        dup = []
        for l, k in enumerate(neigh_j, start=1):
            if l == idx_i_in_j or k <= 0:
                continue
            idx_k_in_i = find_neighbor(ni, k)
            nk = T[k]
            idx_i_in_k = find_neighbor(nk, i)
            idx_j_in_k = find_neighbor(nk, j)
            del nk.neighbor[idx_j_in_k - 1]
            nk.neighbor.insert(idx_j_in_k - 1, i)
            if idx_k_in_i > 0:
                dup.append(k)
                error += merge(P, nk, i, cross=idx_i_in_k > idx_j_in_k)
        lnv, err, phase = eat(P, ni, nj, idx_j_in_i, idx_i_in_j)
        error += err
        psi *= phase
        lnZ += lnv
        for k in dup:
            merge(P, ni, k, cross=False)
            idx = find_neighbor(ni, k)
            if P.cut_bond or (P.Dmax > 0 and ni.mps[idx - 1].shape[1] > P.Dmax):
                error += cut_bondim_opt(tn, i, idx)
        nj.mps.clear()
        nj.neighbor.clear()
        if P.compress:                          # its discarded sum is not added (:694-700)
            compress_opt(P, ni) if P.svdopt else compress(P, ni)
        if P.select in (0, 1):
            count_add_nodes(tn, [i] + ni.neighbor)
        for t in ni.mps:
            tn.maxdim = max(tn.maxdim, t.shape[1])
    for nd in T.values():                       # network_lognorm (:489-501); its sign goes to tn.sign
        if nd.mps and all(s.shape[1] == 1 for s in nd.mps):
            lnZ += math.log(abs(float(nd.mps[0].sum().item())))
    return lnZ, error, psi


# ---------------------------------------------------------------------------
# ising.jl
# ---------------------------------------------------------------------------

def ising_network(n, edges, weights, fields, beta, device="cuda", pos1=0, val1=0, pos2=0, val2=0, **params):
    """``ising_network`` (ising.jl:20-227): one site per incident edge, the
    coupling on the lower-numbered end, the field on the first/leaf site."""
    P = Params(**params)
    dt = torch.float64
    deg = [0] * (n + 1)
    for (i, j) in edges:
        deg[i] += 1
        deg[j] += 1
    nodes = {k: Node() for k in range(1, n + 1)}
    eye = torch.eye(2, dtype=dt)

    def site(node, d, f, Q):
        if d == 1:
            return rs((torch.diag(f) @ Q).sum(0), 1, 2, 1)
        if not node.neighbor:
            return rs((torch.diag(f) @ Q).T.contiguous(), 1, 2, 2)
        if len(node.neighbor) == d - 1:
            return rs(Q.clone(), 2, 2, 1)
        t3 = torch.zeros(2, 2, 2, dtype=dt)
        t3[:, 0, :] = torch.diag(Q[:, 0])
        t3[:, 1, :] = torch.diag(Q[:, 1])
        return t3

    def spins(k):
        s = torch.tensor([1.0, -1.0], dtype=dt)
        if k == pos1:
            s[val1 - 1] = 0.0
        elif k == pos2:
            s[val2 - 1] = 0.0
        return s

    for e, (i, j) in enumerate(edges):
        si, sj = spins(i), spins(j)
        B = torch.exp(beta * float(weights[e]) * torch.outer(si, sj))
        nodes[i].mps.append(site(nodes[i], deg[i], torch.exp(beta * float(fields[i - 1]) * si), B))
        nodes[i].neighbor.append(j)
        nodes[j].mps.append(site(nodes[j], deg[j], torch.exp(beta * float(fields[j - 1]) * sj), eye))
        nodes[j].neighbor.append(i)
    for k in range(1, n + 1):
        if deg[k] == 0:
            hk = float(fields[k - 1])
            nodes[k].mps.append(torch.full((1, 1, 1), math.exp(beta * hk) + math.exp(-beta * hk), dtype=dt))
    for nd in nodes.values():
        nd.mps = [t.to(device) for t in nd.mps]
        nd.cano = len(nd.mps)
    return Network(nodes, P, n, beta)
