"""The workload configurations beyond the batched spin glass, at the reduced
sizes where the FP64 oracle finishes in seconds:

  random-regular +-1 spin glass (n = 60 here; the n = 200 case is frozen in
      tests/golden/rrg200.json) at beta 0.5, 1.0, 1.5, Dmax 32, chi 128;
  Gaussian Ising on an L x L lattice (L = 10 here; 32 in full), h ~ N(0,
      0.2^2), beta 1, Dmax 48, chi 256, differentiated: the adjoint against
      pinning on a 64-edge subset and against central finite differences;
  double-layer norm of a random real PEPS (L = 3..5, D = 2..3; 16 x 16 in
      full) as a generic TensorNetwork of fused tensors, exact against
      sum |psi|^2 of the ket layer and truncated against the oracle.

Bars: identical integer traces and |dlnZ|/n <= 1e-10 against the oracle;
rtol 1e-10 against exact norms; observables within 1e-7 of pinning
(test/test_ising.jl:61-62) and gradients within 1e-7 of central differences.
"""
import numpy as np
import pytest

from oracle import exact as X
from oracle import ising as OI
from oracle import network as ON

pytestmark = pytest.mark.gpu


def fnv(vals):
    h = 2166136261
    for v in vals:
        h = ((h ^ (v & 0xffffffff)) * 16777619) & 0xffffffff
    return h - (1 << 32) if h >= (1 << 31) else h


def rows(tr):
    return [(i, j, int(ri) | (int(rj) << 1), len(d), fnv(d), len(s), fnv(s)) for (i, j, ri, rj, d, s) in tr]


def oracle_trace(build):
    ON.TRACE = []
    tn = build()
    out = ON.contraction(tn)
    tr = ON.TRACE
    ON.TRACE = None
    return out, rows(tr), tn


def test_random_regular_spin_glass_reduced(catn):
    r = np.random.default_rng(60)
    n = 60
    e = X.random_regular_graph(n, 3, r)
    w, h = r.choice([-1.0, 1.0], size=len(e)), r.normal(0, 0.1, n)
    for beta in (0.5, 1.0, 1.5):
        (lz, err, psi), orows, tn = oracle_trace(lambda: OI.ising_network(n, e, w, h, beta, Dmax=32, chi=128))
        net = catn.ising_network(n, e, w, h, beta, Dmax=32, chi=128)
        dlz, derr, dpsi = catn.contraction(net, trace=True)
        assert [tuple(int(x) for x in row[:7]) for row in net.trace] == orows
        assert abs(dlz - lz) / n <= 1e-10
        assert dpsi == psi and net.maxdim_intermediate == tn.maxdim_intermediate


def test_gaussian_lattice_adjoint_reduced(catn):
    """32 x 32 configuration at L = 10: one gradient run against pinning on a
    64-edge subset (one batch of 1 + 4 * 64 pinned networks) and against
    central differences."""
    r = np.random.default_rng(4)
    L = 10
    n = L * L
    e = X.square_edges(L)
    w, h, beta = r.normal(size=len(e)), r.normal(0, 0.2, n), 1.0
    kw = dict(Dmax=48, chi=256)
    lnZ, dw, dh = catn.gradient(catn.ising_network(n, e, w, h, beta, **kw))
    subset = sorted(r.choice(len(e), size=64, replace=False).tolist())
    insts = [dict(n=n, edges=e, weights=w, fields=h, beta=beta)]
    for q in subset:
        m, nn = e[q]
        for v1 in (1, 2):
            for v2 in (1, 2):
                insts.append(dict(n=n, edges=e, weights=w, fields=h, beta=beta, pos1=m, val1=v1, pos2=nn, val2=v2))
    b = catn.IsingBatch(insts, **kw)
    b.run()
    lz = b.lnZ()
    assert lz[0] == pytest.approx(lnZ, abs=1e-10)
    p = np.exp(lz[1:] - lz[0]).reshape(len(subset), 2, 2)
    c_pin = p[:, 0, 0] - p[:, 0, 1] - p[:, 1, 0] + p[:, 1, 1]
    np.testing.assert_allclose(dw[subset] / beta, c_pin, atol=1e-7)
    eps = 1e-5
    for q in subset[:3]:
        wp, wm = w.copy(), w.copy()
        wp[q] += eps
        wm[q] -= eps
        fd = (catn.contraction(catn.ising_network(n, e, wp, h, beta, **kw))[0] -
              catn.contraction(catn.ising_network(n, e, wm, h, beta, **kw))[0]) / (2 * eps)
        assert abs(fd - dw[q]) < 1e-7


@pytest.mark.parametrize("L", [3, 4])
def test_peps_norm_exact(catn, L):
    """Fused double layer, exact mode: <psi|psi> = sum |psi|^2 of the ket layer."""
    from catn_b200 import graphs
    kt, ki, et, ei = graphs.peps_double_layer(L, 2, 2, np.random.default_rng(100 + L))
    ref = float(np.sum(X.exact_contract(kt, ki) ** 2))
    lnZ, err, psi = catn.contraction(catn.TensorNetwork(et, ei, Dmax=-1, chi=100_000))
    assert np.exp(lnZ) * psi == pytest.approx(ref, rel=1e-10)


def test_peps_norm_matrix_free_randomized_swaps(catn, monkeypatch):
    """The fused double-layer PEPS norm with every large swap on the
    randomized route, matrix-free (rsvd = 2: the swap matrix applied from
    the two sites), against the oracle running the reference's randomized
    SVD on the formed matrix with the same sketch; the route's threshold is
    lowered to 12 so that a 4 x 4 PEPS reaches it (16 randomized swaps)."""
    from catn_b200 import graphs
    from oracle import mps as OM
    monkeypatch.setattr(OM, "RSVD_MIN", 12)
    monkeypatch.setattr(OM, "RSVD_SKETCH_SEED", 5)
    monkeypatch.setattr(OM, "RSVD_CALLS", 0)
    _, _, et, ei = graphs.peps_double_layer(4, 2, 2, np.random.default_rng(300))
    (lz, err, psi), orows, tn = oracle_trace(lambda: ON.TensorNetwork.from_tensors(et, ei, Dmax=16, chi=8))
    assert OM.RSVD_CALLS > 0
    net = catn.TensorNetwork(et, ei, Dmax=16, chi=8, rsvd=2, rsvd_min_dim=12, seed=5)
    dlz, derr, dpsi = catn.contraction(net, trace=True)
    assert [tuple(int(x) for x in row[:7]) for row in net.trace] == orows
    assert abs(dlz - lz) <= 1e-10 * max(1.0, abs(lz))
    assert dpsi == psi


@pytest.mark.parametrize("L,D,Dmax,chi", [(4, 2, 8, 16), (5, 2, 8, 16), (4, 3, 16, 32)])
def test_peps_norm_truncated_matches_oracle(catn, L, D, Dmax, chi):
    from catn_b200 import graphs
    _, _, et, ei = graphs.peps_double_layer(L, D, 2, np.random.default_rng(200 + L * D))
    (lz, err, psi), orows, tn = oracle_trace(
        lambda: ON.TensorNetwork.from_tensors(et, ei, Dmax=Dmax, chi=chi))
    net = catn.TensorNetwork(et, ei, Dmax=Dmax, chi=chi)
    dlz, derr, dpsi = catn.contraction(net, trace=True)
    assert [tuple(int(x) for x in row[:7]) for row in net.trace] == orows
    assert abs(dlz - lz) <= 1e-10 * max(1.0, abs(lz))
    assert abs(derr - err) <= 1e-12 + 1e-6 * abs(err)
    assert dpsi == psi
