"""BraKet networks <psi|psi> (reference src/braket.jl): the oracle against
dense exact norms on the reference's own test shapes
(test/test_braket.jl:246-347, real tensors), its invariants and error paths;
the engine compiled for the host (tests/hostcheck) against the oracle; and,
marked gpu, libcatn_b200 against the oracle.

Bars: rtol 1e-10 against the exact norm (the reference's own tolerance,
test/test_braket.jl:256); against the oracle, the edge order identical and
|dlnZ| <= 1e-12, err within 1e-12 + 1e-8 |err|.
"""
import ctypes as ct
import os
import sys

import numpy as np
import pytest

from oracle import braket as B

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "hostcheck"))
import build as hostbuild  # noqa: E402

sys.path.pop(0)

from catn_b200 import _lib as L  # noqa: E402


def chains_and_trees(seed):
    r = np.random.default_rng(seed)
    return [
        ([r.normal(size=(2, 2)), r.normal(size=(2, 2, 2)), r.normal(size=(2, 2))],
         [["p1", "a"], ["a", "p2", "b"], ["b", "p3"]]),
        ([r.normal(size=(2, 3)), r.normal(size=(3, 2, 3)), r.normal(size=(3, 2, 3)), r.normal(size=(3, 2))],
         [["p1", "a"], ["a", "p2", "b"], ["b", "p3", "c"], ["c", "p4"]]),
        ([r.normal(size=(2, 3)), r.normal(size=(3, 2, 3)), r.normal(size=(3, 2, 3)), r.normal(size=(3, 2, 3)),
          r.normal(size=(3, 2))],
         [["p1", "a"], ["a", "p2", "b"], ["b", "p3", "c"], ["c", "p4", "d"], ["d", "p5"]]),
        ([r.normal(size=(2, 2, 2, 2)), r.normal(size=(2, 2)), r.normal(size=(2, 2)), r.normal(size=(2, 2))],
         [["a", "b", "c", "pc"], ["a", "p1"], ["b", "p2"], ["c", "p3"]]),
        ([r.normal(size=(3, 2, 3)), r.normal(size=(2, 3)), r.normal(size=(3, 4, 2, 3)), r.normal(size=(4, 2)),
          r.normal(size=(2, 3))],
         [["a", "p1", "b"], ["p2", "a"], ["b", "c", "p3", "d"], ["c", "p4"], ["p5", "d"]]),
    ]


def oracle_run(ts, ixs, **kw):
    bk = B.braket_network(ts, ixs, **kw)
    B.TRACE = []
    lz, err, psi = B.contraction(bk)
    tr = B.TRACE
    B.TRACE = None
    return lz, err, psi, tr, bk


@pytest.mark.parametrize("svdopt", [True, False])
def test_oracle_norm_matches_exact(svdopt):
    """test/test_braket.jl:246-303 (real-tensor cases)."""
    for ts, ixs in chains_and_trees(123):
        ref = B.exact_norm(ts, ixs)
        lz, err, psi, _, _ = oracle_run(ts, ixs, chi=10_000, svdopt=svdopt)
        assert np.exp(lz) * psi == pytest.approx(ref, rel=1e-10)
        assert ref >= 0


def test_oracle_finite_chi_lossless():
    """test/test_braket.jl:309-316: chi above the Schmidt rank is lossless."""
    r = np.random.default_rng(5)
    ts = [r.normal(size=(2, 2)), r.normal(size=(2, 2, 2)), r.normal(size=(2, 2, 2)), r.normal(size=(2, 2))]
    ixs = [["p1", "a"], ["a", "p2", "b"], ["b", "p3", "c"], ["c", "p4"]]
    lz, _, psi, _, _ = oracle_run(ts, ixs, chi=64)
    assert np.exp(lz) * psi == pytest.approx(B.exact_norm(ts, ixs), rel=1e-8)


def test_oracle_structure_invariants():
    """test/test_braket.jl:318-338: physical legs <= D, junction bond <= d."""
    r = np.random.default_rng(6)
    bk = B.braket_network([r.normal(size=(2, 3)), r.normal(size=(3, 2, 3)), r.normal(size=(3, 2))],
                          [["p1", "a"], ["a", "p2", "b"], ["b", "p3"]], chi=8)
    for node in bk.tensors.values():
        assert all(s.shape[1] <= 3 for s in node.mps)
    node = B.braket_node(r.normal(size=(3, 2, 3, 3)), [10, 20, 30], 2, chi=10_000)
    assert node.mps[2].shape[2] <= 2 and node.mps[3].shape[0] <= 2
    assert all(s.shape[1] <= 3 for s in node.mps)
    assert node.layer == [True] * 3 + [False] * 3 and node.neighbor == [10, 20, 30] * 2


def test_oracle_rejects_cycles_and_bad_labels():
    """test/test_braket.jl:340-345 plus the constructor's error paths."""
    r = np.random.default_rng(7)
    with pytest.raises(ValueError, match="cycle"):
        B.braket_network([r.normal(size=(2, 2, 2))] * 3, [["a", "c", "p1"], ["a", "b", "p2"], ["b", "c", "p3"]])
    with pytest.raises(ValueError, match="physical"):
        B.braket_network([r.normal(size=(2, 2)), r.normal(size=(2, 2))], [["a", "b"], ["a", "b"]])


def loopy_states(seed):
    """Cyclic virtual-bond graphs: a triangle and open PEPS (L_x x L_y, bond D,
    physical 2), the loopy extension's test shapes (the reference rejects
    them, test/test_braket.jl:340-345)."""
    r = np.random.default_rng(seed)
    out = [([r.normal(size=(2, 2, 2)) for _ in range(3)], [["a", "c", "p1"], ["a", "b", "p2"], ["b", "c", "p3"]])]
    for (lx, ly, D) in [(2, 2, 2), (2, 3, 2), (3, 3, 2), (3, 3, 3), (4, 3, 2)]:
        ts, ixs = [], []
        for y in range(ly):
            for x in range(lx):
                ix = ([f"h{x - 1}_{y}"] if x > 0 else []) + ([f"h{x}_{y}"] if x < lx - 1 else []) + \
                     ([f"v{x}_{y - 1}"] if y > 0 else []) + ([f"v{x}_{y}"] if y < ly - 1 else []) + [f"p{x}_{y}"]
                ts.append(r.normal(size=[D] * (len(ix) - 1) + [2]))
                ixs.append(ix)
        out.append((ts, ixs))
    return out


@pytest.mark.parametrize("svdopt", [True, False])
def test_oracle_loopy_norm_matches_exact(svdopt):
    """Loopy extension in exact mode: <psi|psi> of triangles and PEPS against
    the dense norm, at the reference's own tolerance."""
    for ts, ixs in loopy_states(41):
        lz, err, psi, tr, _ = oracle_run(ts, ixs, chi=10_000, svdopt=svdopt, loops=True)
        assert np.exp(lz) * psi == pytest.approx(B.exact_norm(ts, ixs), rel=1e-10)
        assert any(len(t) == 4 for t in tr)


def test_loopy_rejections():
    r = np.random.default_rng(9)
    with pytest.raises(ValueError, match="parallel"):
        B.braket_network([r.normal(size=(2, 2, 2)), r.normal(size=(2, 2, 2))], [["a", "b", "p1"], ["a", "b", "p2"]],
                         loops=True)


@pytest.fixture(scope="module")
def host():
    return ct.CDLL(hostbuild.build())


def _inputs(ts, ixs):
    ids, labels = {}, []
    for ix in ixs:
        for lbl in ix:
            ids.setdefault(lbl, len(ids) + 1)
            labels.append(ids[lbl])
    nd = np.array([t.ndim for t in ts], np.int32)
    dims = np.array([d for t in ts for d in t.shape], np.int64)
    data = np.ascontiguousarray(np.concatenate([np.ravel(t, order="F") for t in ts]))
    return nd, dims, data, np.array(labels, np.int32)


def host_run(lib, ts, ixs, **kw):
    p = L.make_params(Dmax=-1, select=2, reverse=False, **kw)
    nd, dims, data, lab = _inputs(ts, ixs)
    res = L.Result()
    tr = np.zeros(8 * 256, np.int32)
    st = lib.catn_hostcheck_braket(ct.byref(p), ct.c_int(len(ts)), L.ptr(nd), L.ptr(dims), L.ptr(data), L.ptr(lab),
                                   ct.c_longlong(1 << 27), ct.byref(res), L.ptr(tr), ct.c_int(256))
    return st, res, tr[:8 * res.nsteps].reshape(-1, 8)


@pytest.mark.parametrize("kw", [dict(chi=10_000), dict(chi=10_000, svdopt=False), dict(chi=2),
                                dict(chi=3, norm_method=2)])
def test_host_engine_matches_oracle(host, kw):
    for ts, ixs in chains_and_trees(11):
        lz, err, psi, tr, bk = oracle_run(ts, ixs, **kw)
        st, res, dtr = host_run(host, ts, ixs, **kw)
        assert st == 0
        assert [(int(a), int(b)) for a, b in dtr[:, :2]] == [(t[0], t[1]) for t in tr]
        assert abs(res.lnZ - lz) <= 1e-12
        assert abs(res.err - err) <= 1e-12 + 1e-8 * abs(err)
        assert res.psi == psi
        assert res.maxdim == bk.maxdim_intermediate


LOOPY_KW = [dict(chi=10_000), dict(chi=10_000, svdopt=False), dict(chi=4), dict(chi=3, norm_method=2)]


def _loopy_check(lz, err, psi, tr, bk, dlz, derr, dpsi, dtr, maxdim, exact=None):
    assert [(int(a), int(b)) for a, b in dtr[:, :2]] == [(t[0], t[1]) for t in tr]
    assert abs(dlz - lz) <= 1e-10 * max(1.0, abs(lz))
    assert abs(derr - err) <= 1e-10 + 1e-8 * abs(err)
    assert dpsi == psi
    assert maxdim == bk.maxdim_intermediate
    if exact is not None:
        assert np.exp(dlz) * dpsi == pytest.approx(exact, rel=1e-10)


@pytest.mark.parametrize("kw", LOOPY_KW)
def test_host_engine_loopy_matches_oracle(host, kw):
    """Loopy extension: the engine compiled for the host against the oracle's
    restatement, edge order and fused-bond dims included (trace column 4
    counts the fusions of a step)."""
    fused = 0
    for ts, ixs in loopy_states(43):
        lz, err, psi, tr, bk = oracle_run(ts, ixs, loops=True, **kw)
        st, res, dtr = host_run(host, ts, ixs, braket_loops=True, **kw)
        assert st == 0
        _loopy_check(lz, err, psi, tr, bk, res.lnZ, res.err, res.psi, dtr, res.maxdim,
                     B.exact_norm(ts, ixs) if kw["chi"] > 100 else None)
        fused += int(dtr[:, 4].sum())
    assert fused > 0


def test_host_engine_rejects_cycles_without_loops(host):
    ts, ixs = loopy_states(44)[1]
    st, _, _ = host_run(host, ts, ixs, chi=100)
    assert st == L.CATN_EINVAL


@pytest.mark.gpu
@pytest.mark.parametrize("kw", LOOPY_KW)
def test_gpu_loopy_braket_matches_oracle(catn, kw):
    for ts, ixs in loopy_states(45):
        lz, err, psi, tr, bk = oracle_run(ts, ixs, loops=True, **kw)
        net = catn.braket_network(ts, ixs, loops=True, **kw)
        dlz, derr, dpsi = catn.contraction(net, trace=True)
        _loopy_check(lz, err, psi, tr, bk, dlz, derr, dpsi, net.trace, net.maxdim_intermediate,
                     B.exact_norm(ts, ixs) if kw["chi"] > 100 else None)


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(chi=10_000), dict(chi=10_000, svdopt=False), dict(chi=2)])
def test_gpu_braket_matches_oracle_and_exact(catn, kw):
    for ts, ixs in chains_and_trees(21):
        lz, err, psi, tr, bk = oracle_run(ts, ixs, **kw)
        net = catn.braket_network(ts, ixs, **kw)
        dlz, derr, dpsi = catn.contraction(net, trace=True)
        assert [(int(a), int(b)) for a, b in net.trace[:, :2]] == [(t[0], t[1]) for t in tr]
        assert abs(dlz - lz) <= 1e-12
        assert abs(derr - err) <= 1e-12 + 1e-8 * abs(err)
        assert dpsi == psi
        assert net.maxdim_intermediate == bk.maxdim_intermediate
        if kw["chi"] > 100:
            assert np.exp(dlz) * dpsi == pytest.approx(B.exact_norm(ts, ixs), rel=1e-10)


@pytest.mark.gpu
def test_gpu_braket_rejections(catn):
    r = np.random.default_rng(8)
    with pytest.raises(ValueError, match="cycle"):
        catn.braket_network([r.normal(size=(2, 2, 2))] * 3, [["a", "c", "p1"], ["a", "b", "p2"], ["b", "c", "p3"]])
    with pytest.raises(NotImplementedError):
        catn.braket_network([np.ones((2, 2), complex), np.ones((2, 2), complex)], [["p1", "a"], ["a", "p2"]])
    with pytest.raises(ValueError, match="parallel"):
        catn.braket_network([r.normal(size=(2, 2, 2)), r.normal(size=(2, 2, 2))], [["a", "b", "p1"], ["a", "b", "p2"]],
                            loops=True)
