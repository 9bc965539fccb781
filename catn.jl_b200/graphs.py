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
