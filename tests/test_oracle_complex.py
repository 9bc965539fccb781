"""The oracle on complex networks (test/test_complex.jl:7-64 restated): the
cases a complex device path will be pinned against.  The reference contracts
bonds without conjugation (src/mps_node.jl:475) and takes conj(V) only where
the SVD's factors are split (src/tensor_network.jl:365,381)."""
import numpy as np
import pytest

from oracle import exact as X
from oracle import mps as M
from oracle import network as ON


def _crandn(r, *shape):
    return r.normal(size=shape) + 1j * r.normal(size=shape)


def test_eat_of_two_leaves_does_not_conjugate():
    r = np.random.default_rng(1)
    u, v = _crandn(r, 4), _crandn(r, 4)
    ni = M.MPSNode.from_tensor(u, [2], norm_method=0)
    nj = M.MPSNode.from_tensor(v, [1], norm_method=0)
    ln, err, ph = M.eat(ni, nj, 1, 1)
    assert not ni.mps
    assert np.exp(ln) * ph == pytest.approx(np.sum(u * v))
    assert not np.isclose(np.exp(ln) * ph, np.vdot(u, v))


@pytest.mark.parametrize("cut", [ON.cut_bondim, ON.cut_bondim_opt])
def test_cut_keeps_a_complex_low_rank_bond(cut):
    r = np.random.default_rng(2)
    P = _crandn(r, 3, 2) @ _crandn(r, 2, 4)
    Qm = _crandn(r, 4, 2) @ _crandn(r, 2, 3)
    tn = ON.TensorNetwork.from_tensors([P, Qm], [["a", "m"], ["m", "b"]], chi=1000, Dmax=2)
    cut(tn, 1, 2)
    assert tn.tensors[1].mps[1].shape[1] == 2
    got = np.einsum("am,mb->ab", M.mps2raw(tn.tensors[1]), M.mps2raw(tn.tensors[2]))
    np.testing.assert_allclose(got, P @ Qm, atol=1e-8)


@pytest.mark.parametrize("svdopt", [True, False])
def test_finite_dmax_loop_of_rank_two_bonds(svdopt):
    r = np.random.default_rng(3)
    ts = [_crandn(r, 4, 2) @ _crandn(r, 2, 4) for _ in range(4)]
    ixs = [["a", "b"], ["b", "c"], ["c", "d"], ["d", "a"]]
    ref = X.exact_contract(ts, ixs)
    tn = ON.TensorNetwork.from_tensors(ts, ixs, Dmax=2, chi=64, select=1, compress=True, svdopt=svdopt)
    lz, err, psi = ON.contraction(tn)
    assert np.exp(lz) * psi == pytest.approx(ref, rel=1e-6)


@pytest.mark.parametrize("sel", [0, 1, 2])
def test_exact_mode_matches_einsum(sel):
    r = np.random.default_rng(4 + sel)
    nets = [
        ([_crandn(r, 3, 4), _crandn(r, 4, 5), _crandn(r, 5, 3)], [["a", "b"], ["b", "c"], ["c", "a"]]),
        ([_crandn(r, 2, 3, 4), _crandn(r, 2), _crandn(r, 3), _crandn(r, 4)], [["a", "b", "c"], ["a"], ["b"], ["c"]]),
        ([_crandn(r, 2, 3), _crandn(r, 3, 2), _crandn(r, 2, 3), _crandn(r, 3, 2)],
         [["a", "b"], ["b", "c"], ["c", "d"], ["d", "a"]]),
    ]
    for ts, ixs in nets:
        ref = X.exact_contract(ts, ixs)
        tn = ON.TensorNetwork.from_tensors(ts, ixs, Dmax=-1, chi=10_000, select=sel, reverse=True, compress=True,
                                           norm_method=1)
        lz, err, psi = ON.contraction(tn)
        assert np.exp(lz) * psi == pytest.approx(ref, rel=1e-10)
