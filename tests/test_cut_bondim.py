"""cut_bondim! and cut_bondim_opt! called directly on a network before its
contraction (src/tensor_network.jl:342-388, :399-477), against the oracle.

The reference's contraction! only reaches the opt form (through cut_bond);
the plain form is a public function a user calls on a network.  Each cut's
discarded sum is compared with the oracle's (rtol 1e-10), then the cut
network is contracted: the integer trace must be identical and lnZ within
1e-10 relative.  The CPU tests run the engine's host build (team of one
thread, tests/hostcheck); the GPU tests go through the C ABI.
"""
import ctypes as ct
import os
import sys

import numpy as np
import pytest

from oracle import network as ON

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "hostcheck"))
import build as hostbuild  # noqa: E402

sys.path.pop(0)

from catn_b200 import _lib as L  # noqa: E402


def fnv(vals):
    h = 2166136261
    for v in vals:
        h = ((h ^ (v & 0xffffffff)) * 16777619) & 0xffffffff
    return h - (1 << 32) if h >= (1 << 31) else h


def rows(tr):
    return [(i, j, int(ri) | (int(rj) << 1), len(d), fnv(d), len(s), fnv(s)) for (i, j, ri, rj, d, s) in tr]


def grid(L_, D, seed):
    """Closed L x L grid of random tensors with bond dimension D; node
    (r, c) -> id r * L + c + 1, legs in the order right, down, left, up."""
    r = np.random.default_rng(seed)
    ts, ixs = [], []
    for y in range(L_):
        for x in range(L_):
            ix = []
            if x + 1 < L_:
                ix.append(f"h{y}_{x}")
            if y + 1 < L_:
                ix.append(f"v{y}_{x}")
            if x > 0:
                ix.append(f"h{y}_{x - 1}")
            if y > 0:
                ix.append(f"v{y - 1}_{x}")
            ixs.append(ix)
            ts.append(r.normal(size=(D,) * len(ix)))
    return ts, ixs


# (i, idx_j_in_i, opt): corner, centre and edge bonds, the same bond twice.
# A plain cut of two canonical sites can see a fully degenerate spectrum
# (after cut_bondim_opt!(5, 2) the bond 5-4 has four equal singular values):
# which Dmax of them survive is then an arbitrary choice of the SVD, in the
# reference as here, so the cases keep a gap at the cut (checked below).
CUTS = [(1, 1, 0), (5, 2, 1), (2, 1, 0), (5, 4, 0), (9, 1, 1), (1, 1, 1)]
KW = dict(Dmax=3, chi=16)


def cut_gaps(ts, ixs, cuts, Dmax):
    """Relative gap s[Dmax-1] - s[Dmax] of every cut's bond spectrum, on the
    oracle's state just before that cut."""
    from oracle import mps as M
    tn = ON.TensorNetwork.from_tensors(ts, ixs, Dmax=Dmax, chi=16)
    out = []
    for i, k, opt in cuts:
        ni = tn.tensors[i]
        j = ni.neighbor[k - 1]
        nj = tn.tensors[j]
        kj = M.find_neighbor(nj, i)
        if opt:
            M.cano_to(ni, k)
            M.cano_to(nj, kj)
        mats = []
        for A in (ni.mps[k - 1], nj.mps[kj - 1]):
            mats.append(M.rs(np.transpose(A, (0, 2, 1)), A.shape[0] * A.shape[2], A.shape[1]))
        s = np.linalg.svd(mats[0] @ mats[1].T, compute_uv=False)
        out.append((s[Dmax - 1] - s[Dmax]) / s[0] if len(s) > Dmax else 1.0)
        (ON.cut_bondim_opt if opt else ON.cut_bondim)(tn, i, k)
    return out


def oracle_run(ts, ixs, cuts, **kw):
    tn = ON.TensorNetwork.from_tensors(ts, ixs, **kw)
    errs = [(ON.cut_bondim_opt if opt else ON.cut_bondim)(tn, i, k) for i, k, opt in cuts]
    ON.TRACE = []
    out = ON.contraction(tn)
    tr = rows(ON.TRACE)
    ON.TRACE = None
    return errs, out, tr


@pytest.fixture(scope="module")
def host():
    return ct.CDLL(hostbuild.build())


def host_run(lib, ts, ixs, cuts, cut_only, **kw):
    from catn_b200.network import TensorNetwork
    tn = TensorNetwork(ts, ixs, **kw)   # label resolution only
    p = L.make_params(trace=True, **tn.params)
    ndims = np.array([t.ndim for t in tn.tensors], dtype=np.int32)
    dims = np.array([d for t in tn.tensors for d in t.shape], dtype=np.int64)
    data = np.ascontiguousarray(np.concatenate([np.ravel(t, order="F") for t in tn.tensors]))
    nbrs = np.array([v for ix in tn.neighbors for v in ix], dtype=np.int32)
    cl = np.array([v for c in cuts for v in c] or [0], dtype=np.int32)
    res = L.Result()
    cap = 256
    tr = np.zeros(8 * cap, dtype=np.int32)
    lib.catn_hostcheck_dense_cuts.restype = ct.c_int
    st = lib.catn_hostcheck_dense_cuts(ct.byref(p), ct.c_int(tn.n), L.ptr(ndims), L.ptr(dims), L.ptr(data),
                                       L.ptr(nbrs), L.ptr(cl), ct.c_int(len(cuts)), ct.c_int(cut_only),
                                       ct.c_longlong(1 << 28), ct.byref(res), L.ptr(tr), ct.c_int(cap))
    trows = [tuple(int(x) for x in row[:7]) for row in tr[: 8 * min(res.nsteps, cap)].reshape(-1, 8)]
    return st, res, trows


def test_cut_cases_have_a_spectral_gap():
    ts, ixs = grid(3, 4, 11)
    assert min(cut_gaps(ts, ixs, CUTS, KW["Dmax"])) > 1e-2


def test_host_cuts_match_oracle(host):
    ts, ixs = grid(3, 4, 11)
    errs, (lz, err, psi), orows = oracle_run(ts, ixs, CUTS, **KW)
    assert all(e > 0 for e in errs[:5])   # every cut truncates the bond from 4 to 3
    for k in range(len(CUTS)):
        st, res, _ = host_run(host, ts, ixs, CUTS[: k + 1], 1, **KW)
        assert st == 0
        assert res.err == pytest.approx(errs[k], rel=1e-10, abs=1e-13)
        assert res.nsteps == 0
    st, res, trows = host_run(host, ts, ixs, CUTS, 0, **KW)
    assert st == 0
    assert trows == orows
    assert res.lnZ == pytest.approx(lz, rel=1e-10)
    assert res.psi == psi


def test_host_cut_changes_the_contraction(host):
    """The same network without cuts gives another lnZ: the cuts reach the
    contraction."""
    ts, ixs = grid(3, 4, 11)
    _, res_cut, _ = host_run(host, ts, ixs, CUTS[:2], 0, **KW)
    _, res_plain, _ = host_run(host, ts, ixs, [], 0, **KW)
    assert abs(res_cut.lnZ - res_plain.lnZ) > 1e-8


def test_host_cut_of_an_open_leg_is_a_state_error(host):
    """cut_bondim! on an open leg raises in the reference; the engine ends
    the instance with CATN_ESTATE (the C ABI rejects it before launching)."""
    r = np.random.default_rng(3)
    ts = [r.normal(size=(4, 4, 2)), r.normal(size=(4, 4)), r.normal(size=(4, 4))]
    ixs = [["a", "b", "o"], ["b", "c"], ["c", "a"]]
    st, res, _ = host_run(host, ts, ixs, [(1, 3, 0)], 1, Dmax=3, chi=16)
    assert st == 6   # CATN_ESTATE


@pytest.mark.gpu
def test_gpu_cuts_match_oracle(catn):
    ts, ixs = grid(3, 4, 11)
    errs, (lz, err, psi), orows = oracle_run(ts, ixs, CUTS, **KW)
    tn = catn.TensorNetwork(ts, ixs, **KW)
    catn.adapt(catn.B200, tn, trace=True)
    got = [(catn.cut_bondim_opt if opt else catn.cut_bondim)(tn, i, k) for i, k, opt in CUTS]
    assert got == pytest.approx(errs, rel=1e-10, abs=1e-13)
    dlz, derr, dpsi = catn.contraction(tn, trace=True)
    assert [tuple(int(x) for x in row[:7]) for row in tn.trace] == orows
    assert dlz == pytest.approx(lz, rel=1e-10)
    assert dpsi == psi


@pytest.mark.gpu
def test_gpu_cut_boundary_cases(catn):
    r = np.random.default_rng(3)
    ts = [r.normal(size=(4, 4, 2)), r.normal(size=(4, 4)), r.normal(size=(4, 4))]
    ixs = [["a", "b", "o"], ["b", "c"], ["c", "a"]]
    tn = catn.TensorNetwork(ts, ixs, Dmax=3, chi=16)
    with pytest.raises(catn.CatnError):
        catn.cut_bondim(tn, 1, 3)          # open leg: error() in the reference
    with pytest.raises(catn.CatnError):
        catn.cut_bondim(tn, 4, 1)          # no node 4
    e = catn.cut_bondim(tn, 1, 1)          # still usable after the rejected calls
    assert e > 0
    catn.contraction(tn)
    with pytest.raises(ValueError):
        catn.cut_bondim(tn, 1, 1)          # contraction! consumed the network
    exact = catn.TensorNetwork(ts, ixs, Dmax=-1, chi=16)
    assert catn.cut_bondim(exact, 1, 1) == 0.0   # Dmax < 0: a no-op returning 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("opt", [False, True])
def test_gpu_cut_of_a_low_rank_bond_is_exact(catn, opt):
    """test/test_contraction.jl:42-57: a bond of rank 2 stored as dimension
    4, cut to Dmax = 2, keeps the network's value (here the open-leg result
    of contracting it)."""
    r = np.random.default_rng(42)
    P = r.normal(size=(3, 2)) @ r.normal(size=(2, 4))
    Qm = r.normal(size=(4, 2)) @ r.normal(size=(2, 3))
    tn = catn.TensorNetwork([P, Qm], [["a", "m"], ["m", "b"]], chi=1000, Dmax=2)
    err = (catn.cut_bondim_opt if opt else catn.cut_bondim)(tn, 1, 2)
    assert abs(err) < 1e-12 * np.abs(P @ Qm).max()
    lnZ, _, psi = catn.contraction(tn)
    got = catn.result_tensor(tn) * (np.exp(lnZ) * psi)   # the survivor is kept normalised
    ref = P @ Qm
    if got.shape != ref.shape or not np.allclose(got, ref, atol=1e-8):
        got = got.T
    np.testing.assert_allclose(got, ref, atol=1e-8)


@pytest.mark.gpu
def test_gpu_cut_on_an_ising_network_and_gradient_rejection(catn):
    """Cuts apply to Ising networks too (catn_ising_create's MPS form): the
    same cuts on the oracle's Ising network give the same errors and lnZ.  A
    gradient run of a cut network is rejected (the cuts are not taped)."""
    from oracle import exact as X
    from oracle import ising as OI
    r = np.random.default_rng(8)
    L_ = 5
    n = L_ * L_
    e = X.square_edges(L_)
    w, h = r.normal(size=len(e)), r.normal(0, 0.1, n)
    kw = dict(Dmax=1, chi=16)
    cuts = [(7, 1, 1), (13, 2, 1)]
    ref = OI.ising_network(n, e, w, h, 0.7, **kw)
    errs = [ON.cut_bondim_opt(ref, i, k) for i, k, _ in cuts]
    lz, _, _ = ON.contraction(ref)
    net = catn.ising_network(n, e, w, h, 0.7, **kw)
    got = [catn.cut_bondim_opt(net, i, k) for i, k, _ in cuts]
    assert got == pytest.approx(errs, rel=1e-10, abs=1e-13)
    with pytest.raises(catn.CatnError):
        catn.gradient(net)
    assert catn.contraction(net)[0] == pytest.approx(lz, rel=1e-10)


def _random_cuts(ts, ixs, count, seed):
    """`count` random (node, leg, opt) cuts of real bonds with a spectral gap
    at Dmax on the oracle's state (the first seed from `seed` on that has
    one)."""
    nbr_counts = [len(ix) for ix in ixs]
    for s in range(seed, seed + 50):
        r = np.random.default_rng(s)
        cuts = []
        for _ in range(count):
            i = int(r.integers(1, len(ts) + 1))
            cuts.append((i, int(r.integers(1, nbr_counts[i - 1] + 1)), int(r.integers(0, 2))))
        if min(cut_gaps(ts, ixs, cuts, KW["Dmax"])) > 1e-3:
            return cuts
    raise AssertionError("no gapped cut sequence found")


def test_host_random_cut_sequences_match_oracle(host):
    """Twelve random cuts on a closed 4 x 4 grid (bond dimension 4, Dmax 3),
    replayed before the contraction: each cut's discarded sum, then the cut
    network's trace and lnZ, against the oracle."""
    ts, ixs = grid(4, 4, 23)
    cuts = _random_cuts(ts, ixs, 12, 100)
    errs, (lz, err, psi), orows = oracle_run(ts, ixs, cuts, **KW)
    for k in (3, 7, 11):
        st, res, _ = host_run(host, ts, ixs, cuts[: k + 1], 1, **KW)
        assert st == 0
        assert res.err == pytest.approx(errs[k], rel=1e-10, abs=1e-13)
    st, res, trows = host_run(host, ts, ixs, cuts, 0, **KW)
    assert st == 0
    assert trows == orows
    assert res.lnZ == pytest.approx(lz, rel=1e-10)
