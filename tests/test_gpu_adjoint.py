"""GPU tests of the device adjoint through the C ABI (catn_ising_grad,
catn_batch_grad_launch / _results): d lnZ / d w = beta <s_i s_j> and
d lnZ / d h = beta <s_k> against brute force, central finite differences of
the device lnZ, and the reference's pinning definition of magnetization /
correlation (src/ising.jl:263-339) contracted by the same library.

Bars: 1e-12 absolute against brute force (exact mode); 1e-8 absolute against
central differences (step 1e-5) on lossless contractions; against pinning,
1e-7 absolute on the observables at the workload's Dmax = 32, chi = 128
(the reference's own pinned-observable tolerance is rtol 1e-7,
test/test_ising.jl:61-62).
"""
import numpy as np
import pytest

from oracle import exact as X

pytestmark = pytest.mark.gpu


def test_triangle_and_square_against_brute_force(catn):
    e, w, h, b = [(1, 2), (2, 3), (3, 1)], [0.4, 0.6, -0.3], [0.1, -0.2, 0.05], 0.35
    lz, dw, dh = catn.gradient(catn.ising_network(3, e, w, h, b, Dmax=-1, chi=10000))
    m, c = X.brute_observables(3, e, w, h, b)
    np.testing.assert_allclose(dh / b, m, atol=1e-12)
    np.testing.assert_allclose(dw / b, c, atol=1e-12)
    r = np.random.default_rng(5)
    e = X.square_edges(4)
    w, h, b = r.normal(size=len(e)), r.normal(0, 0.3, 16), 0.9
    lz, dw, dh = catn.gradient(catn.ising_network(16, e, w, h, b, Dmax=-1, chi=10000))
    m, c = X.brute_observables(16, e, w, h, b)
    assert lz == pytest.approx(X.brute_lnZ(16, e, w, h, b), rel=1e-12)
    np.testing.assert_allclose(dh / b, m, atol=1e-12)
    np.testing.assert_allclose(dw / b, c, atol=1e-12)


@pytest.mark.parametrize("L,beta,kw", [(6, 0.8, dict(Dmax=-1, chi=100000)), (8, 1.0, dict(Dmax=8, chi=32)),
                                       (6, 0.8, dict(Dmax=1000, chi=100000, cut_bond=True))])
def test_against_central_differences(catn, L, beta, kw):
    r = np.random.default_rng(100 + L)
    e = X.square_edges(L)
    n = L * L
    w, h = r.normal(size=len(e)), r.normal(0, 0.2, n)
    _, dw, dh = catn.gradient(catn.ising_network(n, e, w, h, beta, **kw))

    def lnz(w_, h_):
        return catn.contraction(catn.ising_network(n, e, w_, h_, beta, **kw))[0]

    eps, worst = 1e-5, 0.0
    for q in range(0, len(e), len(e) // 5):
        wp, wm = w.copy(), w.copy()
        wp[q] += eps
        wm[q] -= eps
        worst = max(worst, abs((lnz(wp, h) - lnz(wm, h)) / (2 * eps) - dw[q]))
    for q in range(0, n, n // 5):
        hp, hm = h.copy(), h.copy()
        hp[q] += eps
        hm[q] -= eps
        worst = max(worst, abs((lnz(w, hp) - lnz(w, hm)) / (2 * eps) - dh[q]))
    assert worst < 1e-8


def test_adjoint_matches_pinning_at_workload_settings(catn):
    """One gradient run against the 1 + 2n and 1 + 4|E| pinned contractions."""
    r = np.random.default_rng(8)
    L = 8
    e = X.square_edges(L)
    n = L * L
    w, h, b = r.normal(size=len(e)), r.normal(0, 0.1, n), 1.3
    kw = dict(Dmax=32, chi=128)
    m_pin = catn.magnetization(n, e, w, h, b, **kw)
    c_pin = catn.correlation(n, e, w, h, b, **kw)
    m_adj = catn.magnetization(n, e, w, h, b, method="adjoint", **kw)
    c_adj = catn.correlation(n, e, w, h, b, method="adjoint", **kw)
    np.testing.assert_allclose(m_adj, m_pin, atol=1e-7)
    np.testing.assert_allclose(c_adj, c_pin, atol=1e-7)


def test_batch_gradients_equal_single_network_gradients(catn):
    r = np.random.default_rng(9)
    insts = []
    for q in range(6):
        L = int(r.choice([6, 8, 10]))
        e = X.square_edges(L)
        insts.append(dict(n=L * L, edges=e, weights=r.normal(size=len(e)), fields=r.normal(0, 0.1, L * L),
                          beta=float(r.uniform(0.5, 2.0))))
    out = catn.IsingBatch(insts, Dmax=32, chi=128).grad()
    for d, (lz, dw, dh) in zip(insts, out):
        lz1, dw1, dh1 = catn.gradient(catn.ising_network(d["n"], d["edges"], d["weights"], d["fields"], d["beta"],
                                                         Dmax=32, chi=128))
        assert lz == lz1
        np.testing.assert_array_equal(dw, dw1)
        np.testing.assert_array_equal(dh, dh1)


def test_torch_autograd_function(catn):
    import torch
    r = np.random.default_rng(10)
    e = X.square_edges(4)
    w = torch.tensor(r.normal(size=len(e)), dtype=torch.float64, requires_grad=True)
    h = torch.tensor(r.normal(0, 0.2, 16), dtype=torch.float64, requires_grad=True)
    lz = catn.ising_lnZ(w, h, 16, e, 0.7, Dmax=-1, chi=10000)
    (2.0 * lz).backward()
    m, c = X.brute_observables(16, e, w.detach().numpy(), h.detach().numpy(), 0.7)
    np.testing.assert_allclose(h.grad.numpy(), 2.0 * 0.7 * m, atol=1e-12)
    np.testing.assert_allclose(w.grad.numpy(), 2.0 * 0.7 * c, atol=1e-12)


def test_rejections(catn):
    from catn_b200 import _lib as L
    e = X.square_edges(3)
    with pytest.raises(L.CatnError):
        catn.gradient(catn.ising_network(9, e, np.ones(len(e)), np.zeros(9), 0.5, Dmax=4, chi=8, compress=True))
    tn = catn.ising_network(9, e, np.ones(len(e)), np.zeros(9), 0.5, Dmax=4, chi=8)
    dev = tn._ensure_device()
    lib = L.load()
    res = L.Result()
    dw, dh = np.zeros(len(e)), np.zeros(9)
    assert lib.catn_ising_grad(dev.handle, res, L.ptr(dw), L.ptr(dh), -1) == L.CATN_EINVAL
    assert "ckpt_interval" in L.last_error(lib)


@pytest.mark.parametrize("K", [1, 7, 64])
def test_checkpointed_gradients_equal_whole_tape(catn, K):
    """ckpt_interval K > 0 recomputes K-step segments in the backward pass;
    the values, records and accumulation order are those of the whole tape,
    so lnZ and every gradient entry are equal bit for bit."""
    r = np.random.default_rng(31)
    L = 10
    e = X.square_edges(L)
    n = L * L
    w, h = r.normal(size=len(e)), r.normal(0, 0.2, n)
    tn = catn.ising_network(n, e, w, h, 1.0, Dmax=48, chi=256)
    lz0, dw0, dh0 = catn.gradient(tn, ckpt_interval=0)
    lz, dw, dh = catn.gradient(tn, ckpt_interval=K)
    assert lz == lz0
    np.testing.assert_array_equal(dw, dw0)
    np.testing.assert_array_equal(dh, dh0)


def test_checkpointed_batch_gradients(catn):
    r = np.random.default_rng(32)
    insts = []
    for q in range(5):
        L = int(r.choice([6, 8, 10]))
        e = X.square_edges(L)
        insts.append(dict(n=L * L, edges=e, weights=r.normal(size=len(e)), fields=r.normal(0, 0.1, L * L),
                          beta=float(r.uniform(0.5, 2.0))))
    whole = catn.IsingBatch(insts, Dmax=32, chi=128).grad()
    ckpt = catn.IsingBatch(insts, Dmax=32, chi=128, ckpt_interval=16).grad()
    for (lz0, dw0, dh0), (lz, dw, dh) in zip(whole, ckpt):
        assert lz == lz0
        np.testing.assert_array_equal(dw, dw0)
        np.testing.assert_array_equal(dh, dh0)
