"""The oracle pinned against the reference's own known-answer tests.

The reference ships no golden vectors (its tests draw random inputs), so the
numpy restatement is pinned by restating those tests -- same structure, same
tolerances -- with seeded inputs, plus independent exact checkers (brute
force, row transfer matrix, dense einsum).  Each test cites the reference
test it restates.
"""
import numpy as np
import pytest

from oracle import exact as X
from oracle import ising as OI
from oracle import linalg as LA
from oracle import mps as M
from oracle import network as ON


def rng(seed):
    return np.random.default_rng(seed)


# --- test/test_ising.jl ------------------------------------------------------
def test_chain_transfer_matrix():            # test_ising.jl:17-23
    L, J, b = 6, 0.7, 0.4
    tn = OI.ising_network(L, [(i, i + 1) for i in range(1, L)], [J] * (L - 1), [0.0] * L, b, Dmax=-1, chi=10000)
    assert ON.contraction(tn)[0] == pytest.approx(X.chain_lnZ(L, J, b), rel=1e-9)


def test_triangle_brute_force():             # test_ising.jl:25-43
    e, w, h = [(1, 2), (2, 3), (3, 1)], [0.5, -0.8, 1.1], [0.2, -0.1, 0.4]
    tn = OI.ising_network(3, e, w, h, 0.3, Dmax=-1, chi=10000)
    assert ON.contraction(tn)[0] == pytest.approx(X.brute_lnZ(3, e, w, h, 0.3), rel=1e-9)


def test_magnetization_correlation():        # test_ising.jl:45-66
    e, w, h = [(1, 2), (2, 3), (3, 1)], [0.4, 0.6, -0.3], [0.1, -0.2, 0.05]
    m_ref, c_ref = X.brute_observables(3, e, w, h, 0.35)
    np.testing.assert_allclose(OI.magnetization(3, e, w, h, 0.35, Dmax=-1, chi=10000), m_ref, rtol=1e-7)
    np.testing.assert_allclose(OI.correlation(3, e, w, h, 0.35, Dmax=-1, chi=10000), c_ref, rtol=1e-7)


def test_free_energy_consistency():          # test_ising.jl:68-85
    e, w, h = [(1, 2), (2, 3), (3, 1)], [0.6, -0.5, 0.9], [0.15, -0.3, 0.2]
    lnZ = ON.contraction(OI.ising_network(3, e, w, h, 0.45, Dmax=-1, chi=10000))[0]
    lps, F = OI.free_energy(OI.ising_network(3, e, w, h, 0.45, Dmax=-1, chi=10000))
    assert lps == pytest.approx(lnZ / 3, rel=1e-9)
    assert F == pytest.approx(-lnZ / (3 * 0.45), rel=1e-9)


def test_isolated_spins():                   # test_ising.jl:87-102
    tn = OI.ising_network(1, [], [], [0.5], 0.6, Dmax=-1, chi=10000)
    assert ON.contraction(tn)[0] == pytest.approx(np.log(2 * np.cosh(0.3)), rel=1e-9)
    tn = OI.ising_network(2, [], [], [0.3, 0.7], 0.6, Dmax=-1, chi=10000)
    assert ON.contraction(tn)[0] == pytest.approx(np.log(2 * np.cosh(0.18)) + np.log(2 * np.cosh(0.42)), rel=1e-9)


@pytest.mark.parametrize("L", [3, 4])
def test_square_lattice_brute_force_and_transfer(L):
    r = rng(L)
    e = X.square_edges(L)
    w, h = r.normal(size=len(e)), r.normal(0, 0.1, L * L)
    bf = X.brute_lnZ(L * L, e, w, h, 0.7)
    assert X.square_transfer_lnZ(L, L, e, w, h, 0.7) == pytest.approx(bf, rel=1e-12)
    tn = OI.ising_network(L * L, e, w, h, 0.7, Dmax=-1, chi=100000)
    assert ON.contraction(tn)[0] == pytest.approx(bf, rel=1e-9)


def test_config1_8x8_transfer_matrix():
    """8x8 ferromagnet, beta 0.44, Dmax 20, chi 200 -- the reference's own
    CPU-runnable configuration -- against the exact row transfer matrix."""
    e = X.square_edges(8)
    w, h = np.ones(len(e)), np.zeros(64)
    tn = OI.ising_network(64, e, w, h, 0.44, Dmax=20, chi=200)
    lps, _ = OI.free_energy(tn)
    assert abs(lps - X.square_transfer_lnZ(8, 8, e, w, h, 0.44) / 64) < 1e-12


# --- test/test_contraction.jl --------------------------------------------------
def test_construction_neighbor_order():      # test_contraction.jl:8-18
    r = rng(1)
    A, B, C = r.normal(size=(2, 3)), r.normal(size=(3, 4)), r.normal(size=(4, 2))
    tn = ON.TensorNetwork.from_tensors([A, B, C], [["a", "b"], ["b", "c"], ["c", "a"]], chi=1000)
    assert len(tn.tensors) == 3
    np.testing.assert_allclose(M.mps2raw(tn.tensors[1]), A)
    np.testing.assert_allclose(M.mps2raw(tn.tensors[2]), B)
    assert tn.tensors[1].neighbor == [3, 2]
    assert tn.num_isolated == 0


def test_edge_selection():                   # test_contraction.jl:20-40
    r = rng(2)
    ts = [r.normal(size=(2, 2)), r.normal(size=(2, 2)), r.normal(size=(2, 8)), r.normal(size=(8, 2))]
    tn = ON.TensorNetwork.from_tensors(ts, [["a", "x"], ["x", "y"], ["y", "z"], ["z", "a"]], chi=1000)
    ON.select_edge_init(tn)
    assert set(ON.select_edge_min_dim(tn)) != {3, 4}
    tn = ON.TensorNetwork.from_tensors([r.normal(size=(2, 2)) for _ in range(3)],
                                       [["a", "b"], ["b", "c"], ["c", "a"]], chi=1000)
    assert ON.select_edge_sequentially(tn) == (1, 2)


@pytest.mark.parametrize("cut", [ON.cut_bondim, ON.cut_bondim_opt])
def test_cut_lossless_low_rank(cut):         # test_contraction.jl:42-57
    r = rng(3)
    P = r.normal(size=(3, 2)) @ r.normal(size=(2, 4))
    Q = r.normal(size=(4, 2)) @ r.normal(size=(2, 3))
    tn = ON.TensorNetwork.from_tensors([P, Q], [["a", "m"], ["m", "b"]], chi=1000, Dmax=2)
    cut(tn, 1, 2)
    assert tn.tensors[1].mps[1].shape[1] == 2
    np.testing.assert_allclose(M.mps2raw(tn.tensors[1]) @ M.mps2raw(tn.tensors[2]), P @ Q, atol=1e-8)


def _exact_networks(r):
    return [
        ([r.normal(size=(3, 4)), r.normal(size=(4, 5)), r.normal(size=(5, 3))], [["a", "b"], ["b", "c"], ["c", "a"]]),
        ([r.normal(size=(2, 3, 4)), r.normal(size=2), r.normal(size=3), r.normal(size=4)],
         [["a", "b", "c"], ["a"], ["b"], ["c"]]),
        ([r.normal(size=(2, 3)), r.normal(size=(3, 2)), r.normal(size=(2, 3)), r.normal(size=(3, 2))],
         [["a", "b"], ["b", "c"], ["c", "d"], ["d", "a"]]),
    ]


@pytest.mark.parametrize("sel", [0, 1, 2])
@pytest.mark.parametrize("rev", [False, True])
@pytest.mark.parametrize("comp", [False, True])
def test_exact_mode_matches_einsum(sel, rev, comp):   # test_contraction.jl:69-88
    for ts, ixs in _exact_networks(rng(4)):
        ref = float(X.exact_contract(ts, ixs))
        tn = ON.TensorNetwork.from_tensors(ts, ixs, Dmax=-1, chi=10000, select=sel, reverse=rev, compress=comp)
        lnZ, err, psi = ON.contraction(tn)
        assert np.exp(lnZ) * psi == pytest.approx(ref, rel=1e-8)


def test_finite_dmax_loop():                 # test_contraction.jl:90-96
    r = rng(5)
    ts = [r.normal(size=(4, 4)) for _ in range(4)]
    ixs = [["a", "b"], ["b", "c"], ["c", "d"], ["d", "a"]]
    ref = float(X.exact_contract(ts, ixs))
    lnZ, err, psi = ON.contraction(ON.TensorNetwork.from_tensors(ts, ixs, Dmax=4, chi=64, select=1, compress=True))
    assert np.exp(lnZ) * psi == pytest.approx(ref, rel=1e-6)


# --- test/test_openleg.jl ------------------------------------------------------
def test_open_legs():                        # test_openleg.jl:14-37
    r = rng(6)
    ts = [r.normal(size=(2, 4)), r.normal(size=(4, 2, 4)), r.normal(size=(4, 2))]
    ixs = [["p1", "a"], ["a", "p2", "b"], ["b", "p3"]]
    ref = X.exact_contract(ts, ixs)
    tn = ON.TensorNetwork.from_tensors(ts, ixs, Dmax=-1, chi=10000)
    lnZ, err, psi = ON.contraction(tn)
    got = ON.result_tensor(tn) * (np.exp(lnZ) * psi)
    assert sorted(got.shape) == sorted(ref.shape)
    np.testing.assert_allclose(np.sort(np.abs(got).ravel()), np.sort(np.abs(ref).ravel()), rtol=1e-10)


# --- test/test_mps_node.jl -------------------------------------------------------
@pytest.mark.parametrize("dims", [(4,), (3, 5), (2, 3, 4), (2, 3, 2, 3)])
def test_raw2mps_roundtrip(dims):            # test_mps_node.jl:4-19
    T = rng(7).normal(size=dims)
    node = M.MPSNode.from_tensor(T, list(range(1, len(dims) + 1)), chi=1000)
    assert M.order(node) == len(dims)
    np.testing.assert_allclose(M.mps2raw(node), T, atol=1e-12)


def test_canonicalisation():                 # test_mps_node.jl:21-38
    T = rng(8).normal(size=(2, 3, 4, 2))
    node = M.MPSNode.from_tensor(T, [1, 2, 3, 4], chi=1000)
    ref = M.mps2raw(node)
    for idx in (1, 2, 3, 4, 0):
        M.cano_to(node, idx)
        np.testing.assert_allclose(M.mps2raw(node), ref, atol=1e-12)
    M.left_canonical(node)
    assert node.cano == 4
    for t in node.mps[:3]:
        m = M.rs(t, t.shape[0] * t.shape[1], t.shape[2])
        np.testing.assert_allclose(m.T @ m, np.eye(m.shape[1]), atol=1e-8)


def test_cano_tiny_norm_rank_guard():        # test_mps_node.jl:40-49
    T = rng(9).normal(size=(2, 3, 4, 2)) * 1e-16
    node = M.MPSNode.from_tensor(T, [1, 2, 3, 4], chi=1000, cutoff=0.0)
    node.cutoff = 1e-15
    ref = M.mps2raw(node)
    M.cano_to(node, 1)
    np.testing.assert_allclose(M.mps2raw(node), ref, rtol=1e-8)
    M.cano_to(node, 4)
    np.testing.assert_allclose(M.mps2raw(node), ref, rtol=1e-8)


def test_swap_reverse_move():                # test_mps_node.jl:54-70, 87-93
    T = rng(10).normal(size=(2, 3, 4, 5))
    node = M.MPSNode.from_tensor(T, [10, 20, 30, 40], chi=1000)
    M.swap(node, 2, 3)
    assert node.neighbor == [10, 30, 20, 40]
    np.testing.assert_allclose(M.mps2raw(node), T.transpose(0, 2, 1, 3), atol=1e-10)
    node = M.MPSNode.from_tensor(T, [10, 20, 30, 40], chi=1000)
    M.reverse(node)
    assert node.neighbor == [40, 30, 20, 10]
    np.testing.assert_allclose(M.mps2raw(node), T.transpose(3, 2, 1, 0), atol=1e-10)
    node = M.MPSNode.from_tensor(T, [10, 20, 30, 40], chi=1000)
    M.move2tail(node, 1)
    assert node.neighbor[-1] == 10
    np.testing.assert_allclose(M.mps2raw(node), T.transpose(1, 2, 3, 0), atol=1e-10)
    node = M.MPSNode.from_tensor(T, [10, 20, 30, 40], chi=1000)
    M.swap(node, 3, 2)
    assert node.neighbor == [10, 30, 20, 40]
    np.testing.assert_allclose(M.mps2raw(node), T.transpose(0, 2, 1, 3), atol=1e-10)


def test_neighbor_helpers_and_swap_error():  # test_mps_node.jl:72-85
    node = M.MPSNode.from_tensor(rng(11).normal(size=(2, 2, 2)), [5, 6, 7])
    assert M.find_neighbor(node, 6) == 2 and M.find_neighbor(node, 99) == 0
    M.delete_neighbor(node, 6)
    assert node.neighbor == [5, 7]
    node = M.MPSNode.from_tensor(rng(12).normal(size=(4, 4, 4)), [1, 2, 3], chi=2)
    assert M.swap(node, 1, 2) > 0


@pytest.mark.parametrize("fn", [M.compress, M.compress_opt])
def test_compress_preserves(fn):             # test_mps_node.jl:95-111
    T = rng(13).normal(size=(2, 3, 4, 3, 2))
    node = M.MPSNode.from_tensor(T, [1, 2, 3, 4, 5], chi=1000)
    ref = M.mps2raw(node)
    err = fn(node)
    assert node.cano == 1 and err >= 0.0
    np.testing.assert_allclose(M.mps2raw(node), ref, atol=1e-10)


def test_merge_fused_layout():               # test_mps_node.jl:113-129
    T = rng(14).normal(size=(2, 5, 3))
    node = M.MPSNode.from_tensor(T, [7, 8, 7], chi=1000)
    M.merge(node, 7)
    assert node.neighbor.count(7) == 1
    raw = M.mps2raw(node)
    np.testing.assert_allclose(raw.reshape(raw.shape[0], raw.shape[1], order="F"),
                               M.rs(T.transpose(0, 2, 1), 6, 5), atol=1e-10)


def test_eat_cases():                        # test_mps_node.jl:131-182
    r = rng(15)
    Ti, Tj = r.normal(size=(2, 3, 4)), r.normal(size=(4, 5))
    ni = M.MPSNode.from_tensor(Ti, [1, 2, 3], chi=1000, norm_method=0)
    nj = M.MPSNode.from_tensor(Tj, [3, 4], chi=1000, norm_method=0)
    ln, err, ph = M.eat(ni, nj, M.find_neighbor(ni, 3), M.find_neighbor(nj, 3))
    raw = M.mps2raw(ni) * np.exp(ln)
    exp_ = np.einsum("abc,cd->abd", Ti, Tj)
    np.testing.assert_allclose(np.sort(raw.ravel()), np.sort(exp_.ravel()), atol=1e-8)
    u, v = r.normal(size=3), r.normal(size=3)
    ni = M.MPSNode.from_tensor(u, [2], norm_method=0)
    nj = M.MPSNode.from_tensor(v, [1], norm_method=0)
    ln, err, ph = M.eat(ni, nj, 1, 1)
    assert not ni.mps and np.exp(ln) * ph == pytest.approx(u @ v)
    Ti, Tj = r.normal(size=(2, 4)), r.normal(size=4)
    ni = M.MPSNode.from_tensor(Ti, [5, 9], chi=1000, norm_method=0)
    nj = M.MPSNode.from_tensor(Tj, [9], chi=1000, norm_method=0)
    ln, err, ph = M.eat(ni, nj, 2, 1)
    assert ni.neighbor == [5]
    np.testing.assert_allclose(M.mps2raw(ni).ravel() * np.exp(ln) * ph, Ti @ Tj, atol=1e-8)
    ni = M.MPSNode.from_tensor(r.normal(size=(2, 3, 4)), [1, 2, 3], chi=1000, norm_method=1)
    nj = M.MPSNode.from_tensor(r.normal(size=(4, 5, 6)), [3, 4, 5], chi=1000, norm_method=1)
    M.eat(ni, nj, 3, 1)
    assert ni.cano == len(ni.mps)
    for t in ni.mps[: ni.cano - 1]:
        m = M.rs(t, t.shape[0] * t.shape[1], t.shape[2])
        np.testing.assert_allclose(m.T @ m, np.eye(m.shape[1]), atol=1e-8)


# --- test/test_linalg.jl ---------------------------------------------------------
def test_tsvd_and_rsvd():                    # test_linalg.jl:4-35
    r = rng(16)
    A = r.normal(size=(8, 5))
    U, S, V, _ = LA.tsvd(A)
    np.testing.assert_allclose(U @ np.diag(S) @ V.T, A, atol=1e-12)
    assert np.all(np.diff(S) <= 0)
    U2, S2, V2, _ = LA.tsvd(A, maxdim=2)
    assert S2.size == 2 and np.allclose(S2, S[:2])
    B = U[:, :3] @ np.diag([1.0, 1e-3, 1e-20]) @ V[:, :3].T
    assert LA.tsvd(B, cutoff=1e-10)[1].size == 2
    L = r.normal(size=(50, 4)) @ r.normal(size=(4, 40))
    Ur, Sr, Vr = LA.rsvd(L, 4, 10, 10, rng=np.random.default_rng(0))
    np.testing.assert_allclose(Ur @ np.diag(Sr) @ Vr.T, L, atol=1e-8)
