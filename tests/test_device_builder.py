"""On-device rebuild of Ising site tensors (catn_ising_batch_set_params /
_randomize, csrc/ising_build.cuh): the values of the reference's
ising_network (src/ising.jl:95-183) recomputed from new couplings, fields
and betas on fixed lattices and pins.

CPU (host harness): the recipes the builder records, evaluated with new
parameters, reproduce a host build from those parameters bit for bit and
cover every value of the image; the disorder generator's formula has the
moments of N(0,1).  GPU: networks rebuilt on the device contract to the
lnZ of host-built networks (|dlnZ| <= 1e-12 |lnZ|; the device exp may
differ from the host's in the last bit), with the same step counts.
"""
import ctypes as ct
import os
import sys

import numpy as np
import pytest

from oracle import exact as X

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "hostcheck"))
import build as hostbuild  # noqa: E402

sys.path.pop(0)

from catn_b200 import _lib as L  # noqa: E402


def instances(seed):
    """Square lattices, a triangle with a pendant spin, isolated spins, no
    edges at all, and pinned networks: every site layout and pin case."""
    r = np.random.default_rng(seed)
    out = []
    for Lside in (3, 4, 5):
        e = X.square_edges(Lside)
        n = Lside * Lside
        out.append(dict(n=n, edges=e, weights=r.normal(size=len(e)), fields=r.normal(0, 0.3, n),
                        beta=float(r.uniform(0.3, 1.5))))
    tri = [(1, 2), (2, 3), (3, 1), (3, 4)]
    out.append(dict(n=6, edges=tri, weights=r.normal(size=4), fields=r.normal(0, 0.5, 6), beta=0.7))
    out.append(dict(n=3, edges=[], weights=[], fields=r.normal(0, 0.5, 3), beta=0.9))
    e = X.square_edges(4)
    out.append(dict(n=16, edges=e, weights=r.normal(size=len(e)), fields=r.normal(0, 0.3, 16), beta=1.1,
                    pos1=6, val1=1))
    out.append(dict(n=16, edges=e, weights=r.normal(size=len(e)), fields=r.normal(0, 0.3, 16), beta=0.8,
                    pos1=2, val1=2, pos2=11, val2=1))
    return out


def packed(insts):
    n_nodes = np.array([d["n"] for d in insts], np.int32)
    node_off = np.concatenate([[0], np.cumsum(n_nodes)]).astype(np.int64)
    ne = [len(d["edges"]) for d in insts]
    edge_off = np.concatenate([[0], np.cumsum(ne)]).astype(np.int64)
    edges = np.concatenate([np.asarray(d["edges"], np.int32).reshape(-1) for d in insts if len(d["edges"])])
    w = np.concatenate([np.asarray(d["weights"], float) for d in insts])
    h = np.concatenate([np.asarray(d["fields"], float) for d in insts])
    b = np.array([d["beta"] for d in insts], float)
    pins = np.array([[d.get("pos1", 0), d.get("val1", 0), d.get("pos2", 0), d.get("val2", 0)] for d in insts],
                    np.int32).reshape(-1)
    return n_nodes, node_off, edge_off, np.ascontiguousarray(edges), w, h, b, pins


@pytest.fixture(scope="module")
def host():
    lib = ct.CDLL(hostbuild.build())
    lib.catn_hostcheck_ising_recipes.restype = ct.c_longlong
    lib.catn_hostcheck_disorder_normal.restype = ct.c_double
    lib.catn_hostcheck_disorder_normal.argtypes = [ct.c_ulonglong, ct.c_ulonglong, ct.c_ulonglong]
    return lib


def test_recipes_rebuild_the_host_image_exactly(host):
    insts = instances(1)
    n_nodes, node_off, edge_off, edges, w, h, b, pins = packed(insts)
    r = np.random.default_rng(2)
    w2, h2, b2 = r.normal(size=w.size), r.normal(0, 0.4, h.size), r.uniform(0.2, 2.0, b.size)
    p = L.make_params(Dmax=8, chi=32)
    md, cov, tot = ct.c_double(), ct.c_longlong(), ct.c_longlong()
    nrec = host.catn_hostcheck_ising_recipes(ct.byref(p), len(insts), L.ptr(n_nodes), L.ptr(node_off),
                                             L.ptr(edge_off), L.ptr(edges), L.ptr(w), L.ptr(h), L.ptr(b), L.ptr(w2),
                                             L.ptr(h2), L.ptr(b2), L.ptr(pins), ct.byref(md), ct.byref(cov),
                                             ct.byref(tot))
    assert nrec > 0
    assert md.value == 0.0
    assert cov.value == tot.value
    # one recipe per site: two per edge plus one per degree-0 spin
    deg0 = sum(int(np.sum(np.bincount(np.asarray(d["edges"], int).reshape(-1), minlength=d["n"] + 1)[1:] == 0))
               if len(d["edges"]) else d["n"] for d in insts)
    assert nrec == 2 * int(edge_off[-1]) + deg0


def test_disorder_generator_moments(host):
    z = np.array([host.catn_hostcheck_disorder_normal(7, 0, i) for i in range(100_000)])
    y = np.array([host.catn_hostcheck_disorder_normal(7, 1, i) for i in range(100_000)])
    assert abs(z.mean()) < 0.015 and abs(z.var() - 1.0) < 0.02
    assert abs(np.mean(z ** 3)) < 0.05 and abs(np.mean(z ** 4) - 3.0) < 0.1
    assert abs(np.corrcoef(z, y)[0, 1]) < 0.015
    assert abs(np.corrcoef(z[:-1], z[1:])[0, 1]) < 0.015
    assert host.catn_hostcheck_disorder_normal(7, 0, 12345) == z[12345]
    assert host.catn_hostcheck_disorder_normal(8, 0, 12345) != z[12345]


def _close(a, b):
    for x, y in zip(a, b):
        assert x.status == 0 and y.status == 0
        assert abs(x.lnZ - y.lnZ) <= 1e-12 * max(1.0, abs(y.lnZ))
        assert x.nsteps == y.nsteps
        assert x.maxdim == y.maxdim


@pytest.mark.gpu
def test_set_params_matches_host_built_networks(catn):
    insts = instances(3)
    kw = dict(Dmax=8, chi=32)
    bat = catn.IsingBatch(insts, **kw)
    ref = [L.Result.from_buffer_copy(x) for x in bat.run()]
    _, _, _, _, w, h, b, _ = packed(insts)
    # the creation parameters, rebuilt on the device
    bat.set_params(w, h, b)
    bat.launch()
    _close([L.Result.from_buffer_copy(x) for x in bat.fetch()], ref)
    # new disorder and temperatures against a batch built from them on the host
    r = np.random.default_rng(4)
    w2, h2, b2 = r.normal(size=w.size), r.normal(0, 0.4, h.size), r.uniform(0.2, 2.0, b.size)
    bat.set_params(w2, h2, b2)
    bat.launch()
    got = [L.Result.from_buffer_copy(x) for x in bat.fetch()]
    fresh = []
    o_e, o_n = 0, 0
    for q, d in enumerate(insts):
        ne = len(d["edges"])
        fresh.append(dict(d, weights=w2[o_e:o_e + ne], fields=h2[o_n:o_n + d["n"]], beta=float(b2[q])))
        o_e += ne
        o_n += d["n"]
    ref2 = catn.IsingBatch(fresh, **kw).run()
    _close(got, ref2)
    wb, hb, bb = bat.params()
    np.testing.assert_array_equal(wb, w2)
    np.testing.assert_array_equal(hb, h2)
    np.testing.assert_array_equal(bb, b2)
    assert bat.param_bytes == 8 * (w.size + h.size + b.size)
    # gradients need the creation parameters; upload restores them
    with pytest.raises(L.CatnError):
        bat.grad_launch()
    bat.upload()
    bat.launch()
    _close([L.Result.from_buffer_copy(x) for x in bat.fetch()], ref)
    bat.grad()


@pytest.mark.gpu
def test_device_disorder_generation(catn):
    lib = ct.CDLL(hostbuild.build())
    lib.catn_hostcheck_disorder_normal.restype = ct.c_double
    lib.catn_hostcheck_disorder_normal.argtypes = [ct.c_ulonglong, ct.c_ulonglong, ct.c_ulonglong]
    insts = instances(5)
    kw = dict(Dmax=8, chi=32)
    bat = catn.IsingBatch(insts, **kw)
    bat.upload()
    bat.randomize(2024, sigma_w=1.0, sigma_h=0.1)
    bat.launch()
    got = [L.Result.from_buffer_copy(x) for x in bat.fetch()]
    w, h, b = bat.params()
    ew = np.array([lib.catn_hostcheck_disorder_normal(2024, 0, i) for i in range(w.size)])
    eh = 0.1 * np.array([lib.catn_hostcheck_disorder_normal(2024, 1, i) for i in range(h.size)])
    np.testing.assert_allclose(w, ew, rtol=1e-14, atol=1e-15)
    np.testing.assert_allclose(h, eh, rtol=1e-14, atol=1e-15)
    fresh = []
    o_e, o_n = 0, 0
    for q, d in enumerate(insts):
        ne = len(d["edges"])
        fresh.append(dict(d, weights=w[o_e:o_e + ne], fields=h[o_n:o_n + d["n"]], beta=float(b[q])))
        o_e += ne
        o_n += d["n"]
    _close(got, catn.IsingBatch(fresh, **kw).run())
    with pytest.raises(L.CatnError):
        bat.randomize(1, sigma_w=-1.0)
