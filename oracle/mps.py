"""Per-tensor MPS engine (oracle; test infrastructure).

Restates ``src/mps_node.jl`` of CATN.jl.  Sites are ``(left, phys, right)``
numpy arrays; all reshapes are column-major so that flattened indices agree
with Julia's.  Positions are 1-based in every public function, as in the
reference.
"""
import math

import numpy as np

from .linalg import tsvd, rsvd, thin_qr, counter_normal, _svd_full

# Randomized-SVD route of swap! (test infrastructure).  RSVD_MIN overrides
# the reference's size thresholds (7000 / 20000 become RSVD_MIN / 3 RSVD_MIN,
# as the engine's catn_params.rsvd_min_dim does).  RSVD_SKETCH_SEED, when set,
# draws the sketch from the engine's counter-based generator (that seed,
# stream 16 + RSVD_CALLS), which pins the engine's rsvd = 1 mode; callers
# reset RSVD_CALLS to 0 before each network.
RSVD_MIN = None
RSVD_SKETCH_SEED = None
RSVD_CALLS = 0


def svd_full_topk(M, k):
    """The exact top-k singular triplets (all of them when fewer)."""
    U, S, V = _svd_full(M)
    kk = min(k, S.shape[0])
    return U[:, :kk], S[:kk], V[:, :kk]

# Optional step log: list of tuples (op, d0, d1, d2, d3, kept).
STEP_LOG = None


def _log(*rec):
    if STEP_LOG is not None:
        STEP_LOG.append(rec)


def rs(a, *shape):
    """Column-major reshape (Julia ``reshape``)."""
    return np.reshape(a, shape, order="F")


class MPSNode:
    """``MPSNode{T,AT}`` (mps_node.jl:1-29)."""

    def __init__(self, mps, neighbor, cano, chi, cutoff=1e-15, norm_method=1,
                 svdopt=True, swapopt=True):
        self.mps = list(mps)
        self.neighbor = list(neighbor)
        self.cano = int(cano)
        self.chi = int(chi)
        self.cutoff = float(cutoff)
        self.norm_method = int(norm_method)
        self.svdopt = bool(svdopt)
        self.swapopt = bool(swapopt)

    @classmethod
    def from_tensor(cls, tensor, neighbor, chi=32, cutoff=1e-15, norm_method=1,
                    svdopt=True, swapopt=True):
        """``MPSNode(tensor, neighbor; ...)`` (mps_node.jl:23-29)."""
        mps = raw2mps(np.asarray(tensor), chi, cutoff)
        return cls(mps, neighbor, len(mps), chi, cutoff, norm_method, svdopt, swapopt)

    def copy(self):
        return MPSNode([t.copy() for t in self.mps], self.neighbor, self.cano, self.chi,
                       self.cutoff, self.norm_method, self.svdopt, self.swapopt)


def raw2mps(tensor, chi, cutoff):
    """Sequential SVD of a dense tensor into MPS sites (mps_node.jl:31-50)."""
    nd = tensor.ndim
    if nd == 0:
        return []
    dims = tensor.shape
    if nd == 1:
        return [rs(tensor, 1, dims[0], 1)]
    mps = []
    R = rs(tensor, 1, *dims)
    dleft = 1
    for i in range(nd - 1):
        M = rs(R, dleft * dims[i], R.size // (dleft * dims[i]))
        U, S, V, _ = tsvd(M, cutoff=cutoff, maxdim=chi, tag="raw2mps")
        c = S.shape[0]
        mps.append(rs(U, dleft, dims[i], c))
        R = rs(S[:, None] * V.conj().T, c, *dims[i + 1:])
        dleft = c
    mps.append(rs(R, dleft, dims[nd - 1], 1))
    return mps


def mps2raw(node):
    """Dense tensor of a node (mps_node.jl:52-70); legs in site order."""
    mps = node.mps
    if not mps:
        return np.ones(())
    A = mps[0]
    cur = rs(A, A.shape[1], A.shape[2])
    pdim = A.shape[1]
    physdims = [A.shape[1]]
    for B in mps[1:]:
        r, p, r2 = B.shape
        res = cur @ rs(B, r, p * r2)
        pdim *= p
        cur = rs(res, pdim, r2)
        physdims.append(p)
    return rs(cur, *physdims)


def order(node):
    return len(node.mps)


def shape(node):
    return [t.shape[1] for t in node.mps]


def cano_to(node, idx):
    """Move the canonical centre with SVD sweeps (mps_node.jl:72-104).

    The SVD itself runs with cutoff 0; the kept count is then
    ``count(S > node.cutoff)``, falling back to *all* values when none pass.
    """
    if idx == 0:
        idx = len(node.mps)
    if node.cano == idx:
        return node
    if node.cano < idx:
        for i in range(node.cano, idx):            # i = cano .. idx-1 (1-based)
            t = node.mps[i - 1]
            dl, d, dr = t.shape
            U, S, V, _ = tsvd(rs(t, dl * d, dr), cutoff=0.0, tag="cano_r")
            nkeep = int(np.count_nonzero(S > node.cutoff))
            nkeep = S.shape[0] if nkeep == 0 else nkeep
            U, S, V = U[:, :nkeep], S[:nkeep], V[:, :nkeep]
            _log("cano_r", dl, d, dr, 0, nkeep)
            node.mps[i - 1] = rs(U, dl, d, nkeep)
            R = S[:, None] * V.conj().T
            node.mps[i] = np.einsum("ij,jab->iab", R, node.mps[i])
            node.cano = i + 1
    else:
        for i in range(node.cano, idx, -1):        # i = cano .. idx+1
            t = node.mps[i - 1]
            dl, d, dr = t.shape
            Mt = rs(np.transpose(t, (1, 2, 0)), d * dr, dl)
            U, S, V, _ = tsvd(Mt, cutoff=0.0, tag="cano_l")
            nkeep = int(np.count_nonzero(S > node.cutoff))
            nkeep = S.shape[0] if nkeep == 0 else nkeep
            U, S, V = U[:, :nkeep], S[:nkeep], V[:, :nkeep]
            _log("cano_l", dl, d, dr, 0, nkeep)
            node.mps[i - 1] = np.transpose(rs(U, d, dr, nkeep), (2, 0, 1))
            R = S[:, None] * V.conj().T                     # (nkeep, dl)
            node.mps[i - 2] = np.einsum("abc,cd->abd", node.mps[i - 2], R.T)
            node.cano = i - 1
    return node


def left_canonical(node):
    """``left_canonical!`` (mps_node.jl:106)."""
    node.cano = 1
    return cano_to(node, len(node.mps))


def swap(node, i, j):
    """Swap adjacent sites ``i`` and ``j`` with chi truncation (mps_node.jl:126-178).

    Returns the sum of discarded singular values.
    """
    mps = node.mps
    assert abs(i - j) == 1, "swap!: i and j must be consecutive indices"
    assert 1 <= i <= len(mps) and 1 <= j <= len(mps), "swap!: indices out of range"
    if node.cano != i and node.cano != j:
        target = i if abs(node.cano - i) < abs(node.cano - j) else j
        cano_to(node, target)
    tl, tr = (mps[i - 1], mps[j - 1]) if i < j else (mps[j - 1], mps[i - 1])
    d0, d1, d2, d3 = tl.shape[0], tr.shape[1], tl.shape[1], tr.shape[2]
    W = np.einsum("ijk,kab->iajb", tl, tr)
    M = rs(W, d0 * d1, d2 * d3)
    rows, cols = M.shape
    rmin, rbig = (7000, 20000) if RSVD_MIN is None else (RSVD_MIN, 3 * RSVD_MIN)
    if node.swapopt and ((rows > rmin and cols > rmin) or rows > rbig or cols > rbig):
        p = min(cols, 10 * node.chi)
        if RSVD_SKETCH_SEED is None:
            U, S, V = rsvd(M, node.chi, 10, 10)
        elif rows >= p:
            global RSVD_CALLS
            G = counter_normal(RSVD_SKETCH_SEED, 16 + RSVD_CALLS, np.arange(cols * p)).reshape(p, cols).T
            RSVD_CALLS += 1
            U, S, V = rsvd(M, node.chi, 10, 10, sketch=G)
        else:   # the engine takes the exact top-chi subspace for a sketch wider than M
            U, S, V = svd_full_topk(M, node.chi)
        err = 0.0
    else:
        U, S, V, err = tsvd(M, cutoff=node.cutoff, maxdim=node.chi, tag="swap")
    myd = S.shape[0]
    _log("swap", d0, d1, d2, d3, myd)
    if i < j:
        mps[i - 1] = rs(U, d0, d1, myd)
        mps[j - 1] = rs(S[:, None] * V.conj().T, myd, d2, d3)
    else:
        mps[j - 1] = rs(U * S[None, :], d0, d1, myd)
        mps[i - 1] = rs(V.conj().T, myd, d2, d3)
    node.cano = j
    nb = node.neighbor
    nb[i - 1], nb[j - 1] = nb[j - 1], nb[i - 1]
    return err


def move(node, a, b):
    """``move!`` (mps_node.jl:186-199)."""
    err = 0.0
    if a == b:
        return err
    if b > a:
        for idx in range(a, b):
            err += swap(node, idx, idx + 1)
    else:
        for idx in range(a, b, -1):
            err += swap(node, idx, idx - 1)
    return err


def move2tail(node, idx):
    """``move2tail!`` (mps_node.jl:208-217)."""
    err = 0.0
    n = len(node.mps)
    if idx == n:
        cano_to(node, n)
        return err
    for k in range(idx, n):
        err += swap(node, k, k + 1)
    cano_to(node, n)
    return err


def move2head(node, idx):
    """``move2head!`` (mps_node.jl:225-229)."""
    err = move(node, idx, 1)
    cano_to(node, 1)
    return err


def reverse(node):
    """``reverse!`` (mps_node.jl:238-244)."""
    if len(node.mps) <= 1:
        return node
    node.mps = [np.transpose(t, (2, 1, 0)) for t in node.mps[::-1]]
    node.neighbor.reverse()
    node.cano = len(node.mps) + 1 - node.cano
    return node


def find_neighbor(node, j):
    """1-based position of ``j`` in ``node.neighbor`` or 0 (mps_node.jl:257-260)."""
    try:
        return node.neighbor.index(j) + 1
    except ValueError:
        return 0


def add_neighbor(node, n, pos=0):
    """``add_neighbor!`` (mps_node.jl:267-274)."""
    if pos == 0:
        node.neighbor.append(n)
    else:
        node.neighbor.insert(pos - 1, n)
    return node


def delete_neighbor(node, n):
    """``delete_neighbor!`` (mps_node.jl:282-287)."""
    idx = find_neighbor(node, n)
    if idx == 0:
        raise ValueError(f"delete_neighbor!: neighbor {n} not found")
    del node.neighbor[idx - 1]
    return idx


def logdim(node, idx=None):
    """Sum of log2(phys dim) over sites, or of one site (mps_node.jl:299-311).

    The sum is a left fold, as Julia's ``sum`` over a generator.
    """
    if idx is not None:
        return math.log2(float(node.mps[idx - 1].shape[1]))
    s = 0.0
    first = True
    for t in node.mps:
        v = math.log2(float(t.shape[1]))
        s = v if first else s + v
        first = False
    return s


def lognorm(node):
    """``(log|z|, sign z)`` of a scalar node (mps_node.jl:319-328)."""
    if not node.mps:
        return 0.0, 1.0
    if len(node.mps) == 1 and node.mps[0].shape[1] == 1:
        z = np.sum(node.mps[0])
        return math.log(abs(z)), (z / abs(z) if z != 0 else 0.0)
    raise ValueError("lognorm: computing norm of a non-scalar MPS is not supported in contraction")


def clear(node):
    """``clear!`` (mps_node.jl:335-339)."""
    node.mps.clear()
    node.neighbor.clear()
    return node


def compress(node):
    """``compress!``: left-canonicalise then R->L two-site truncation (mps_node.jl:356-376)."""
    err = 0.0
    if not node.mps:
        return err
    left_canonical(node)
    mps = node.mps
    for j in range(len(mps), 1, -1):
        i = j - 1
        tl, tr = mps[i - 1], mps[j - 1]
        d0, d1 = tl.shape[0], tl.shape[1]
        d2, d3 = tr.shape[1], tr.shape[2]
        mat = rs(np.einsum("ijk,kab->ijab", tl, tr), d0 * d1, d2 * d3)
        U, S, V, e = tsvd(mat, cutoff=node.cutoff, maxdim=node.chi, tag="compress")
        err += e
        myd = S.shape[0]
        _log("compress", d0, d1, d2, d3, myd)
        mps[i - 1] = rs(U * S[None, :], d0, d1, myd)
        mps[j - 1] = rs(V.conj().T, myd, d2, d3)
    node.cano = 1
    return err


def compress_opt(node):
    """``compress_opt!``: QR pre-reduction before each two-site SVD (mps_node.jl:394-447)."""
    err = 0.0
    if not node.mps:
        return err
    left_canonical(node)
    mps = node.mps
    for j in range(len(mps), 1, -1):
        i = j - 1
        tl, tr = mps[i - 1], mps[j - 1]
        d0, d1 = tl.shape[0], tl.shape[1]
        d2, d3 = tr.shape[1], tr.shape[2]
        dd = tl.shape[2]
        matl = rs(tl, d0 * d1, dd)
        matr = rs(tr, dd, d2 * d3)
        flag_left = matl.shape[0] > matl.shape[1]
        if flag_left:
            Ql, Rl = thin_qr(matl)
        else:
            Rl = matl
        flag_right = matr.shape[0] < matr.shape[1]
        if flag_right:
            Qr, Rr = thin_qr(matr.conj().T)
        else:
            Rr = matr.conj().T
        mat = Rl @ Rr.conj().T
        U, S, V, e = tsvd(mat, cutoff=node.cutoff, maxdim=node.chi, tag="compress_opt")
        err += e
        myd = S.shape[0]
        _log("compress_opt", d0, d1, d2, d3, myd)
        U = U * S[None, :]
        if flag_left:
            U = Ql @ U
        if flag_right:
            V = Qr @ V
        mps[i - 1] = rs(U, d0, d1, myd)
        mps[j - 1] = rs(V.conj().T, myd, d2, d3)
    node.cano = 1
    return err


def _norm(node, t):
    if node.norm_method == 1:
        return float(np.linalg.norm(t.reshape(-1)))
    if node.norm_method == 2:
        return float(np.max(np.abs(t)))
    return 1.0


def eat(node, nodej, idx, idxi):
    """Contract leg ``idx`` of ``node`` with leg ``idxi`` of ``nodej`` (mps_node.jl:463-575).

    Returns ``(lognorm, error, phase)``.
    """
    err = 0.0
    one = np.ones((), dtype=node.mps[0].dtype)[()] if node.mps else 1.0
    # case (a): both leaves (mps_node.jl:469-489)
    if len(node.mps) == 1:
        assert len(nodej.mps) == 1
        vi = node.mps[0].reshape(-1, order="F")
        vj = nodej.mps[0].reshape(-1, order="F")
        r = np.sum(vi * vj)
        absr = abs(r)
        _log("eat_a", vi.shape[0], 0, 0, 0, 0)
        if absr <= node.cutoff:
            node.mps.clear()
            del node.neighbor[idx - 1]
            return 0.0, 0.0, one
        lnv = math.log(absr)
        node.mps.clear()
        del node.neighbor[idx - 1]
        return lnv, 0.0, r / absr
    err += move2tail(node, idx)
    last = node.mps[-1]
    mati = rs(last, last.shape[0], last.shape[1])
    # case (b): nodej is a leaf (mps_node.jl:498-528)
    if len(nodej.mps) == 1:
        tj = nodej.mps[0]
        matj = rs(tj, tj.shape[1], 1)
        mat = mati @ matj
        new_tensor = np.einsum("ijk,ka->ija", node.mps[-2], mat)
        _log("eat_b", *node.mps[-2].shape, mati.shape[1], 0)
        nrm = _norm(node, new_tensor)
        node.mps[-2] = new_tensor
        node.cano = node.cano - 1
        node.mps.pop()
        node.neighbor.pop()
        if nrm <= node.cutoff:
            return 0.0, err, one
        node.mps[-1] = node.mps[-1] / nrm
        return math.log(nrm), err, one
    # case (c): general (mps_node.jl:533-574)
    err += move2head(nodej, idxi)
    h = nodej.mps[0]
    matj = rs(h, h.shape[1], h.shape[2])
    mat = mati @ matj
    _log("eat_c", *node.mps[-2].shape, mati.shape[1], matj.shape[1])
    node.mps[-2] = np.einsum("ijk,ka->ija", node.mps[-2], mat)
    node.mps.pop()
    node.cano = len(node.mps)
    node.mps.extend(nodej.mps[1:])
    node.neighbor.pop()
    node.neighbor.extend(nodej.neighbor[1:])
    cano_to(node, len(node.mps))
    center = node.mps[node.cano - 1]
    nrm = _norm(node, center)
    if nrm <= node.cutoff:
        return 0.0, err, one
    node.mps[node.cano - 1] = center / nrm
    return math.log(nrm), err, one


def merge(node, j, cross=False):
    """Fuse the two sites whose neighbour is ``j`` (mps_node.jl:595-622)."""
    positions = [k + 1 for k, v in enumerate(node.neighbor) if v == j]
    if len(positions) != 2:
        raise ValueError(f"merge!: expected exactly 2 sites with neighbor {j}, found {len(positions)}")
    idx1, idx2 = positions
    target = idx1 if cross else idx1 + 1
    err = move(node, idx2, target)
    del node.neighbor[target - 1]
    cano_to(node, idx1)
    a, b = node.mps[idx1 - 1], node.mps[idx1]
    dl, dr2 = a.shape[0], b.shape[2]
    fused = np.einsum("ijk,kab->ijab", a, b)
    _log("merge", dl, a.shape[1], b.shape[1], dr2, 0)
    node.mps[idx1 - 1] = rs(fused, dl, a.shape[1] * b.shape[1], dr2)
    del node.mps[idx1]
    cano_to(node, idx1)
    return err
