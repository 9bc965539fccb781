"""The reference's randomized-SVD route of swap! (mps_node.jl:154-156,
linalg_utils.jl:44-58) with a reproducible sketch (catn_params.rsvd = 1):
the engine draws the Gaussian sketch from its counter-based generator
keyed by (seed, call index), and the oracle, given the same sketch, runs the
reference's algorithm.  With catn_params.rsvd = 2 the engine runs the same
algorithm matrix-free: the products with the swap matrix are applied from
the two sites, the matrix itself is never formed.  The route's size threshold is lowered through
catn_params.rsvd_min_dim (engine) and RSVD_MIN (oracle) so that small
networks reach it; the default thresholds are the reference's 7000 / 20000.

Bars: the per-step integer trace identical to the oracle's and
|dlnZ|/n <= 1e-10; the oracle's sketch generator equal to the engine's
within 1 ulp of the math library.
"""
import ctypes as ct
import os
import sys

import numpy as np
import pytest

from oracle import exact as X
from oracle import linalg as OL
from oracle import mps as OM

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "hostcheck"))
import build as hostbuild  # noqa: E402

sys.path.pop(0)
from test_hostcheck_engine import oracle_ising, run_ising  # noqa: E402

# (name, L, params, route threshold): sketches as wide as the matrix
# (p = n), and a network whose 32 x 32 swap gets a narrow one (p = 10 chi = 20)
CASES = [("full_sketch", 6, dict(Dmax=8, chi=4), 4), ("narrow_sketch", 8, dict(Dmax=32, chi=2), 8)]


def route(monkeypatch, rmin):
    monkeypatch.setattr(OM, "RSVD_MIN", rmin)
    monkeypatch.setattr(OM, "RSVD_SKETCH_SEED", 3)
    monkeypatch.setattr(OM, "RSVD_CALLS", 0)


def instance(L, seed):
    r = np.random.default_rng(seed)
    e = X.square_edges(L)
    return L * L, e, r.normal(size=len(e)), r.normal(0, 0.2, L * L), 0.9


def oracle_run(n, e, w, h, beta, kw):
    OM.RSVD_CALLS = 0
    (lz, err, psi), rows, tn = oracle_ising(n, e, w, h, beta, **kw)
    return lz, rows, OM.RSVD_CALLS


def test_oracle_generator_matches_the_engine_formula():
    lib = ct.CDLL(hostbuild.build())
    lib.catn_hostcheck_disorder_normal.restype = ct.c_double
    lib.catn_hostcheck_disorder_normal.argtypes = [ct.c_ulonglong] * 3
    z = OL.counter_normal(3, 16, np.arange(2000))
    c = np.array([lib.catn_hostcheck_disorder_normal(3, 16, i) for i in range(2000)])
    np.testing.assert_allclose(z, c, rtol=4e-16, atol=4e-16)


def test_oracle_sketched_rsvd_is_exact_with_a_full_sketch():
    r = np.random.default_rng(1)
    A = r.normal(size=(40, 30)) @ np.diag(0.7 ** np.arange(30)) @ r.normal(size=(30, 30))
    G = OL.counter_normal(3, 16, np.arange(30 * 30)).reshape(30, 30).T
    U, S, V = OL.rsvd(A, 5, 10, 10, sketch=G)
    Se = np.linalg.svd(A, compute_uv=False)[:5]
    np.testing.assert_allclose(S, Se, rtol=1e-12)
    np.testing.assert_allclose(np.abs(U.T @ U), np.eye(5), atol=1e-12)


@pytest.mark.parametrize("mode", [1, 2], ids=["formed", "matrix_free"])
@pytest.mark.parametrize("name,L,kw,rmin", CASES, ids=[c[0] for c in CASES])
def test_host_engine_matches_oracle(monkeypatch, name, L, kw, rmin, mode):
    route(monkeypatch, rmin)
    lib = ct.CDLL(hostbuild.build())
    n, e, w, h, beta = instance(L, 7)
    lz, rows, calls = oracle_run(n, e, w, h, beta, kw)
    assert calls > 0   # the route was taken
    st, res, drows = run_ising(lib, n, e, w, h, beta, rsvd=mode, rsvd_min_dim=rmin, seed=3, **kw)
    assert st == 0
    assert drows == rows
    assert abs(res.lnZ - lz) / n <= 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [1, 2], ids=["formed", "matrix_free"])
@pytest.mark.parametrize("name,L,kw,rmin", CASES, ids=[c[0] for c in CASES])
def test_gpu_matches_oracle(monkeypatch, catn, name, L, kw, rmin, mode):
    route(monkeypatch, rmin)
    n, e, w, h, beta = instance(L, 7)
    lz, rows, calls = oracle_run(n, e, w, h, beta, kw)
    assert calls > 0
    tn = catn.ising_network(n, e, w, h, beta, rsvd=mode, rsvd_min_dim=rmin, seed=3, **kw)
    dlz, err, psi = catn.contraction(tn, trace=True)
    drows = [tuple(int(x) for x in r[:7]) for r in tn.trace]
    assert drows == rows
    assert abs(dlz - lz) / n <= 1e-10
    assert err == 0.0 or err >= 0.0
    # rsvd = 0 on the same route: the exact top-chi subspace
    tn0 = catn.ising_network(n, e, w, h, beta, rsvd=0, rsvd_min_dim=rmin, seed=3, **kw)
    lz0 = catn.contraction(tn0)[0]
    assert np.isfinite(lz0)
