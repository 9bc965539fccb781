"""Independent exact checkers (oracle; test infrastructure).

* ``brute_lnZ`` / ``brute_observables``: enumeration over 2^n spin states
  (the reference's ``test/test_ising.jl:130-160`` and
  ``examples/double_layer_ising.jl:120-135`` formulas), n <= 24.
* ``square_transfer_lnZ``: exact row transfer matrix for an L x W open square
  lattice with arbitrary couplings and fields (2^W states per row), the exact
  equivalent of brute force for the 8 x 8 lattice.
* ``chain_lnZ``: open chain transfer matrix (test/test_ising.jl:5-12).
* ``exact_contract``: dense einsum of a whole labelled network
  (test/exact.jl:4-19), output labels in first-seen order.
* graph generators used by the workloads: ``square_edges`` (the reference's
  edge order, examples/double_layer_ising.jl:110-117) and a seeded random
  regular graph.
"""
import itertools
import math

import numpy as np
from scipy.special import logsumexp


def grid_id(r, c, L):
    return (r - 1) * L + c


def square_edges(L, W=None):
    """Open square lattice edges, row-major ids, right then down (1-based)."""
    W = L if W is None else W
    e = []
    for r in range(1, L + 1):
        for c in range(1, W + 1):
            if c < W:
                e.append(((r - 1) * W + c, (r - 1) * W + c + 1))
            if r < L:
                e.append(((r - 1) * W + c, r * W + c))
    return e


def _energies(n, edges, w, h):
    states = ((np.arange(2 ** n)[:, None] >> np.arange(n)[None, :]) & 1) * 2 - 1
    E = states @ np.asarray(h, dtype=float)
    for e, (i, j) in enumerate(edges):
        E = E + w[e] * states[:, i - 1] * states[:, j - 1]
    return states, E


def brute_lnZ(n, edges, w, h, beta):
    """log sum_s exp(beta (sum_e w_e s_i s_j + sum_k h_k s_k)) by enumeration."""
    assert n <= 24, "brute force limited to n <= 24"
    _, E = _energies(n, edges, w, h)
    return float(logsumexp(beta * E))


def brute_observables(n, edges, w, h, beta):
    """(<s_k>, <s_i s_j> per edge) by enumeration."""
    assert n <= 22
    states, E = _energies(n, edges, w, h)
    lw = beta * E
    p = np.exp(lw - logsumexp(lw))
    m = p @ states
    c = np.array([p @ (states[:, i - 1] * states[:, j - 1]) for (i, j) in edges])
    return m, c


def chain_lnZ(L, J, beta):
    T = np.array([[math.exp(beta * J), math.exp(-beta * J)],
                  [math.exp(-beta * J), math.exp(beta * J)]])
    v = np.ones(2)
    return math.log(v @ np.linalg.matrix_power(T, L - 1) @ v)


def square_transfer_lnZ(L, W, edges, w, h, beta):
    """Exact lnZ of an L x W open square lattice by row transfer (any couplings).

    ``edges``/``w`` follow ``square_edges(L, W)``'s node numbering; each edge
    is classified as horizontal (same row) or vertical (next row).
    """
    nstate = 2 ** W
    bits = ((np.arange(nstate)[:, None] >> np.arange(W)[None, :]) & 1) * 2 - 1   # (S, W)
    hmat = np.zeros((L, W))
    vmat = np.zeros((L, W))
    hfield = np.asarray(h, dtype=float).reshape(L, W)
    for e, (i, j) in enumerate(edges):
        ri, ci = divmod(i - 1, W)
        rj, cj = divmod(j - 1, W)
        if ri == rj:
            assert cj == ci + 1
            hmat[ri, ci] += w[e]
        else:
            assert rj == ri + 1 and cj == ci
            vmat[ri, ci] += w[e]

    def row_energy(r):
        E = bits @ hfield[r]
        for c in range(W - 1):
            E = E + hmat[r, c] * bits[:, c] * bits[:, c + 1]
        return E

    logv = beta * row_energy(0)                  # log weights over row-0 states
    for r in range(1, L):
        inter = beta * (bits * vmat[r - 1][None, :]) @ bits.T      # (S_prev, S_next)
        logv = logsumexp(logv[:, None] + inter, axis=0) + beta * row_energy(r)
    return float(logsumexp(logv))


def exact_contract(tensors, ixs):
    """Dense contraction of a labelled network (test/exact.jl:4-19)."""
    counts, order = {}, []
    for ix in ixs:
        for l in ix:
            if l not in counts:
                order.append(l)
            counts[l] = counts.get(l, 0) + 1
    letters = {}
    alphabet = itertools.chain("abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ")
    for l in order:
        letters[l] = next(alphabet)
    out = "".join(letters[l] for l in order if counts[l] == 1)
    spec = ",".join("".join(letters[l] for l in ix) for ix in ixs) + "->" + out
    return np.einsum(spec, *tensors, optimize="greedy")


def random_regular_graph(n, d, rng):
    """Seeded random d-regular simple graph by the configuration model with
    restarts (1-based edge list, each edge (i, j) with i < j, sorted)."""
    for _ in range(1000):
        stubs = np.repeat(np.arange(1, n + 1), d)
        rng.shuffle(stubs)
        pairs = stubs.reshape(-1, 2)
        ok = True
        seen = set()
        for a, b in pairs:
            if a == b:
                ok = False
                break
            key = (min(a, b), max(a, b))
            if key in seen:
                ok = False
                break
            seen.add(key)
        if ok:
            return sorted((int(a), int(b)) for a, b in seen)
    raise RuntimeError("random_regular_graph: no simple graph found")
