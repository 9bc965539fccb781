"""GPU parity tests: libcatn_b200 (through its C ABI) against the oracle and
the exact checkers.  Cases follow the reference's own tests
(test/test_ising.jl, test/test_contraction.jl, test/test_openleg.jl,
test/test_gpu.jl) plus the workload configurations.

Tolerances: the device engine computes in FP64, so lnZ is held to
|dlnZ|/n <= 1e-10 against the FP64 oracle and exact answers at rtol 1e-9
(the reference's own Ising tolerance, test/test_ising.jl:19,39); the integer
edge trace must be identical.
"""
import numpy as np
import pytest

from oracle import exact as X
from oracle import ising as OI
from oracle import network as ON

pytestmark = pytest.mark.gpu


def oracle_run(n, e, w, h, beta, **kw):
    ON.TRACE = []
    tn = OI.ising_network(n, e, w, h, beta, **kw)
    lnZ, err, psi = ON.contraction(tn)
    tr = ON.TRACE
    ON.TRACE = None
    return lnZ, err, psi, tr, tn


def fnv(vals):
    h = 2166136261
    for v in vals:
        h = ((h ^ (v & 0xffffffff)) * 16777619) & 0xffffffff
    return h - (1 << 32) if h >= (1 << 31) else h


def oracle_trace_rows(tr):
    return [(i, j, int(ri) | (int(rj) << 1), len(d), fnv(d), len(s), fnv(s)) for (i, j, ri, rj, d, s) in tr]


def device_rows(tn):
    return [tuple(int(x) for x in r[:7]) for r in tn.trace]


def test_ising_chain_transfer_matrix(catn):
    L, J, b = 6, 0.7, 0.4
    tn = catn.ising_network(L, [(i, i + 1) for i in range(1, L)], [J] * (L - 1), [0.0] * L, b, Dmax=-1, chi=10000)
    lnZ, _, _ = catn.contraction(tn)
    assert lnZ == pytest.approx(X.chain_lnZ(L, J, b), rel=1e-9)


def test_ising_triangle_brute_force(catn):
    edges = [(1, 2), (2, 3), (3, 1)]
    w, h = [0.5, -0.8, 1.1], [0.2, -0.1, 0.4]
    tn = catn.ising_network(3, edges, w, h, 0.3, Dmax=-1, chi=10000)
    lnZ, _, _ = catn.contraction(tn)
    assert lnZ == pytest.approx(X.brute_lnZ(3, edges, w, h, 0.3), rel=1e-9)


def test_isolated_spins(catn):
    tn = catn.ising_network(2, [], [], [0.3, 0.7], 0.6, Dmax=-1, chi=10000)
    lnZ, _, _ = catn.contraction(tn)
    assert lnZ == pytest.approx(np.log(2 * np.cosh(0.18)) + np.log(2 * np.cosh(0.42)), rel=1e-9)


def test_free_energy_consistency(catn):
    edges = [(1, 2), (2, 3), (3, 1)]
    w, h = [0.6, -0.5, 0.9], [0.15, -0.3, 0.2]
    lnZ, _, _ = catn.contraction(catn.ising_network(3, edges, w, h, 0.45, Dmax=-1, chi=10000))
    lps, F = catn.free_energy(catn.ising_network(3, edges, w, h, 0.45, Dmax=-1, chi=10000))
    assert lps == pytest.approx(lnZ / 3, rel=1e-9)
    assert F == pytest.approx(-lnZ / (3 * 0.45), rel=1e-9)


def test_magnetization_correlation_brute_force(catn):
    edges = [(1, 2), (2, 3), (3, 1)]
    w, h = [0.4, 0.6, -0.3], [0.1, -0.2, 0.05]
    m_ref, c_ref = X.brute_observables(3, edges, w, h, 0.35)
    m = catn.magnetization(3, edges, w, h, 0.35, Dmax=-1, chi=10000)
    c = catn.correlation(3, edges, w, h, 0.35, Dmax=-1, chi=10000)
    np.testing.assert_allclose(m, m_ref, rtol=1e-7)
    np.testing.assert_allclose(c, c_ref, rtol=1e-7)


@pytest.mark.parametrize("L,beta,Dmax,chi", [(4, 0.7, -1, 100000), (8, 0.44, 20, 200), (8, 1.0, 8, 32),
                                             (10, 1.0, 32, 128)])
def test_square_spin_glass_matches_oracle(catn, L, beta, Dmax, chi):
    rng = np.random.default_rng(100 + L)
    e = X.square_edges(L)
    w = rng.normal(size=len(e)) if Dmax != 20 else np.ones(len(e))
    h = rng.normal(0, 0.1, L * L) if Dmax != 20 else np.zeros(L * L)
    lz, err, psi, tr, ref = oracle_run(L * L, e, w, h, beta, Dmax=Dmax, chi=chi)
    tn = catn.ising_network(L * L, e, w, h, beta, Dmax=Dmax, chi=chi)
    lnZ, derr, dpsi = catn.contraction(tn, trace=True)
    assert device_rows(tn) == oracle_trace_rows(tr)
    assert abs(lnZ - lz) / (L * L) <= 1e-10
    assert dpsi == psi
    assert tn.maxdim_intermediate == ref.maxdim_intermediate
    assert abs(derr - err) <= 1e-12 + 1e-6 * abs(err)
    ex = X.square_transfer_lnZ(L, L, e, w, h, beta)
    if Dmax < 0:
        assert lnZ == pytest.approx(ex, rel=1e-9)


def test_config1_ferromagnet_8x8(catn):
    """8x8 open ferromagnet, beta 0.44, Dmax 20, chi 200: lnZ/site against the
    exact row transfer matrix (brute force over 2^64 states is infeasible)."""
    e = X.square_edges(8)
    w, h = np.ones(len(e)), np.zeros(64)
    tn = catn.ising_network(64, e, w, h, 0.44, Dmax=20, chi=200, cutoff=1e-15, select=1, norm_method=1)
    lps, F = catn.free_energy(tn)
    ex = X.square_transfer_lnZ(8, 8, e, w, h, 0.44) / 64
    assert abs(lps - ex) <= 1e-10
    assert F == pytest.approx(-lps / 0.44, rel=1e-12)


def _exact_networks(rng):
    return [
        ([rng.normal(size=(3, 4)), rng.normal(size=(4, 5)), rng.normal(size=(5, 3))], [["a", "b"], ["b", "c"], ["c", "a"]]),
        ([rng.normal(size=(2, 3, 4)), rng.normal(size=2), rng.normal(size=3), rng.normal(size=4)],
         [["a", "b", "c"], ["a"], ["b"], ["c"]]),
        ([rng.normal(size=(2, 3)), rng.normal(size=(3, 2)), rng.normal(size=(2, 3)), rng.normal(size=(3, 2))],
         [["a", "b"], ["b", "c"], ["c", "d"], ["d", "a"]]),
    ]


@pytest.mark.parametrize("sel", [0, 1, 2])
@pytest.mark.parametrize("rev", [False, True])
@pytest.mark.parametrize("comp", [False, True])
def test_exact_mode_matches_einsum(catn, sel, rev, comp):
    """test/test_contraction.jl:69-88 -- exact mode equals dense contraction."""
    rng = np.random.default_rng(11)
    for ts, ixs in _exact_networks(rng):
        ref = float(X.exact_contract(ts, ixs))
        tn = catn.TensorNetwork(ts, ixs, Dmax=-1, chi=10000, select=sel, reverse=rev, compress=comp, norm_method=1)
        lnZ, err, psi = catn.contraction(tn)
        assert np.exp(lnZ) * psi == pytest.approx(ref, rel=1e-8)


def test_finite_dmax_loop(catn):
    """test/test_contraction.jl:90-96."""
    rng = np.random.default_rng(12)
    ts = [rng.normal(size=(4, 4)) for _ in range(4)]
    ixs = [["a", "b"], ["b", "c"], ["c", "d"], ["d", "a"]]
    ref = float(X.exact_contract(ts, ixs))
    tn = catn.TensorNetwork(ts, ixs, Dmax=4, chi=64, select=1, compress=True)
    lnZ, err, psi = catn.contraction(tn)
    assert np.exp(lnZ) * psi == pytest.approx(ref, rel=1e-6)


def test_open_legs_result_tensor(catn):
    """test/test_openleg.jl:14-26: result equals the dense contraction up to leg order."""
    rng = np.random.default_rng(13)
    ts = [rng.normal(size=(2, 4)), rng.normal(size=(4, 2, 4)), rng.normal(size=(4, 2))]
    ixs = [["p1", "a"], ["a", "p2", "b"], ["b", "p3"]]
    ref = X.exact_contract(ts, ixs)
    tn = catn.TensorNetwork(ts, ixs, Dmax=-1, chi=10000)
    lnZ, err, psi = catn.contraction(tn)
    got = catn.result_tensor(tn) * (np.exp(lnZ) * psi)
    assert sorted(got.shape) == sorted(ref.shape)
    np.testing.assert_allclose(np.sort(np.abs(got).ravel()), np.sort(np.abs(ref).ravel()), rtol=1e-10)


def test_closed_network_result_tensor_is_one(catn):
    rng = np.random.default_rng(14)
    ts = [rng.normal(size=(2, 3)), rng.normal(size=(3, 4)), rng.normal(size=(4, 2))]
    tn = catn.TensorNetwork(ts, [["a", "b"], ["b", "c"], ["c", "a"]], Dmax=-1, chi=10000)
    catn.contraction(tn)
    r = catn.result_tensor(tn)
    assert r.ndim == 0 and float(r) == 1.0


def test_batch_spin_glass_instances_match_oracle(catn):
    """Uneven-size batch (L in {8..16}) in one persistent launch against the oracle."""
    rng = np.random.default_rng(21)
    insts = []
    for q in range(10):
        L = int(rng.choice([8, 10, 12, 14, 16]))
        e = X.square_edges(L)
        insts.append(dict(n=L * L, edges=e, weights=rng.normal(size=len(e)), fields=rng.normal(0, 0.1, L * L),
                          beta=float(rng.uniform(0.5, 2.0))))
    b = catn.IsingBatch(insts, Dmax=32, chi=128)
    res = b.run()
    for d, r in zip(insts, res):
        lz, err, psi, tr, _ = oracle_run(d["n"], d["edges"], d["weights"], d["fields"], d["beta"], Dmax=32, chi=128)
        assert r.status == 0
        assert r.nsteps == len(tr)
        assert abs(r.lnZ - lz) / d["n"] <= 1e-10
