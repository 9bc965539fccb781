"""Graph builders for Ising / spin-glass workloads.

``square_edges`` reproduces the reference's square-lattice edge order
(examples/double_layer_ising.jl:110-117: row-major node ids, for each site
the right neighbour then the one below, 1-based).  ``random_regular_graph``
is a seeded configuration-model generator (the reference ships none).
"""
import numpy as np


def square_edges(L, W=None):
    W = L if W is None else W
    e = []
    for r in range(1, L + 1):
        for c in range(1, W + 1):
            if c < W:
                e.append(((r - 1) * W + c, (r - 1) * W + c + 1))
            if r < L:
                e.append(((r - 1) * W + c, r * W + c))
    return e


def random_regular_graph(n, d, rng):
    """Random simple d-regular graph on nodes 1..n (sorted (i, j), i < j)."""
    for _ in range(1000):
        stubs = np.repeat(np.arange(1, n + 1), d)
        rng.shuffle(stubs)
        seen = set()
        ok = True
        for a, b in stubs.reshape(-1, 2):
            key = (min(a, b), max(a, b))
            if a == b or key in seen:
                ok = False
                break
            seen.add(key)
        if ok:
            return sorted((int(a), int(b)) for a, b in seen)
    raise RuntimeError("random_regular_graph: no simple graph found")


def spinglass_batch(count, seed, sizes=(8, 10, 12, 14, 16), beta_range=(0.5, 2.0), field_sigma=0.1):
    """Seeded batch of open L x L Gaussian spin glasses (J ~ N(0,1),
    h ~ N(0, field_sigma^2), beta ~ U[beta_range], L uniform over sizes)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        L = int(rng.choice(list(sizes)))
        e = square_edges(L)
        out.append(dict(n=L * L, edges=e, weights=rng.normal(size=len(e)), fields=rng.normal(0, field_sigma, L * L),
                        beta=float(rng.uniform(*beta_range))))
    return out


def peps_double_layer(L, D, d, rng):
    """Random real PEPS on an L x L open lattice and its double-layer norm
    network: site tensor A[p, N, S, W, E] (virtual legs present only towards
    existing neighbours, in that order), E = sum_p A (x) A with each ket leg
    fused with its bra copy into one leg of size D^2 (ket index fastest).

    Returns (ket_tensors, ket_ixs, E_tensors, E_ixs); labels are tuples
    ("v", r, c) / ("h", r, c) for bonds and ("p", r, c) for physical legs.
    The same construction as the reference's PEPS example
    (examples/peps_norm.jl:71-81, 95-113) for real entries.
    """
    ket_t, ket_ix, e_t, e_ix = [], [], [], []
    for r in range(1, L + 1):
        for c in range(1, L + 1):
            bonds = []
            if r > 1:
                bonds.append(("v", r - 1, c))
            if r < L:
                bonds.append(("v", r, c))
            if c > 1:
                bonds.append(("h", r, c - 1))
            if c < L:
                bonds.append(("h", r, c))
            deg = len(bonds)
            A = rng.normal(size=(d,) + (D,) * deg)
            ket_t.append(A)
            ket_ix.append([("p", r, c)] + bonds)
            amat = np.reshape(A, (d, D ** deg), order="F")
            m2 = amat.T @ amat                                  # (alpha, beta)
            t = np.reshape(m2, (D,) * (2 * deg), order="F")     # (l1..ldeg, l1'..ldeg')
            perm = [a for k in range(deg) for a in (k, deg + k)]
            e_t.append(np.reshape(np.transpose(t, perm), (D * D,) * deg, order="F"))
            e_ix.append(bonds)
    return ket_t, ket_ix, e_t, e_ix
