"""The device adjoint (csrc/adjoint.cuh) compiled for the host (team of one
thread, tests/hostcheck): d lnZ / d w and d lnZ / d h against brute-force
beta <s_i s_j>, beta <s_k> and against central finite differences of the
same engine's lnZ (step 1e-5, FP64).

Bars: 1e-12 absolute against brute force in exact mode; 1e-8 absolute
against central differences wherever the contraction's truncation is below
1e-12 per spin (the finite difference's own error is ~1e-10 here).  Where a
cut truly discards singular values, the adjoint treats the discarded part as
zero and agrees with the finite difference only to the truncation level; that
regime is checked against pinning instead (GPU tests).
"""
import ctypes as ct
import os
import subprocess
import sys
import zlib

import numpy as np
import pytest

from oracle import exact as X

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "hostcheck"))
import build as hostbuild  # noqa: E402

sys.path.pop(0)

from catn_b200 import _lib as L  # noqa: E402


@pytest.fixture(scope="module")
def host():
    return ct.CDLL(hostbuild.build())


def grad(lib, n, e, w, h, beta, pins=(0, 0, 0, 0), arena=1 << 28, **kw):
    p = L.make_params(**kw)
    E = np.ascontiguousarray(np.array(e, dtype=np.int32).reshape(-1)) if len(e) else np.zeros(2, np.int32)
    W = np.ascontiguousarray(np.array(w, dtype=np.float64)) if len(w) else np.zeros(1)
    H = np.ascontiguousarray(np.array(h, dtype=np.float64))
    dw = np.zeros(max(len(e), 1))
    dh = np.zeros(n)
    res = L.Result()
    st = lib.catn_hostcheck_ising_grad(ct.byref(p), ct.c_int(n), ct.c_int(len(e)), L.ptr(E), L.ptr(W), L.ptr(H),
                                       ct.c_double(beta), *[ct.c_int(x) for x in pins], ct.c_longlong(arena),
                                       ct.byref(res), L.ptr(dw), L.ptr(dh))
    return st, res.lnZ, dw[:len(e)], dh


def fd_check(lib, n, e, w, h, beta, dw, dh, every=5, eps=1e-5, **kw):
    """Max |adjoint - central difference| over a spread of edges and spins."""
    w, h = np.asarray(w, float), np.asarray(h, float)
    worst = 0.0
    for q in range(0, len(e), max(1, len(e) // every)):
        wp, wm = w.copy(), w.copy()
        wp[q] += eps
        wm[q] -= eps
        fd = (grad(lib, n, e, wp, h, beta, **kw)[1] - grad(lib, n, e, wm, h, beta, **kw)[1]) / (2 * eps)
        worst = max(worst, abs(fd - dw[q]))
    for q in range(0, n, max(1, n // every)):
        hp, hm = h.copy(), h.copy()
        hp[q] += eps
        hm[q] -= eps
        fd = (grad(lib, n, e, w, hp, beta, **kw)[1] - grad(lib, n, e, w, hm, beta, **kw)[1]) / (2 * eps)
        worst = max(worst, abs(fd - dh[q]))
    return worst


def test_triangle_against_brute_force(host):
    e, w, h, b = [(1, 2), (2, 3), (3, 1)], [0.4, 0.6, -0.3], [0.1, -0.2, 0.05], 0.35
    st, lz, dw, dh = grad(host, 3, e, w, h, b, Dmax=-1, chi=10000)
    m, c = X.brute_observables(3, e, w, h, b)
    assert st == 0
    assert lz == pytest.approx(X.brute_lnZ(3, e, w, h, b), rel=1e-12)
    np.testing.assert_allclose(dh / b, m, atol=1e-12)
    np.testing.assert_allclose(dw / b, c, atol=1e-12)


@pytest.mark.parametrize("norm_method", [0, 1, 2])
@pytest.mark.parametrize("select", [0, 1, 2])
def test_square4_exact_against_brute_force(host, norm_method, select):
    r = np.random.default_rng(10 * norm_method + select)
    e = X.square_edges(4)
    w, h, b = r.normal(size=len(e)), r.normal(0, 0.3, 16), 0.8
    st, lz, dw, dh = grad(host, 16, e, w, h, b, Dmax=-1, chi=10000, norm_method=norm_method, select=select)
    m, c = X.brute_observables(16, e, w, h, b)
    assert st == 0
    np.testing.assert_allclose(dh / b, m, atol=1e-12)
    np.testing.assert_allclose(dw / b, c, atol=1e-12)


def test_random_regular_against_brute_force(host):
    r = np.random.default_rng(4)
    e = X.random_regular_graph(14, 3, r)
    w, h, b = r.choice([-1.0, 1.0], size=len(e)), r.normal(0, 0.1, 14), 1.0
    st, _, dw, dh = grad(host, 14, e, w, h, b, Dmax=-1, chi=10000)
    m, c = X.brute_observables(14, e, w, h, b)
    assert st == 0
    np.testing.assert_allclose(dh / b, m, atol=1e-12)
    np.testing.assert_allclose(dw / b, c, atol=1e-12)


def test_isolated_spins_and_pins(host):
    # degree-0 spins: <s> = tanh(beta h)
    st, _, _, dh = grad(host, 2, [], [], [0.3, -0.7], 0.6, Dmax=-1, chi=100)
    assert st == 0
    np.testing.assert_allclose(dh, 0.6 * np.tanh(0.6 * np.array([0.3, -0.7])), atol=1e-14)
    # pinned network: gradient of the pinned lnZ, against finite differences
    e, w, h = [(1, 2), (2, 3), (3, 1), (3, 4)], [0.4, 0.6, -0.3, 0.8], [0.1, -0.2, 0.05, 0.3]
    for pins in [(1, 1, 0, 0), (2, 2, 4, 1)]:
        st, _, dw, dh = grad(host, 4, e, w, h, 0.7, pins=pins, Dmax=-1, chi=100)
        assert st == 0
        assert fd_check(host, 4, e, w, h, 0.7, dw, dh, pins=pins, Dmax=-1, chi=100) < 1e-8


CASES = [
    ("sq6_exact", 6, 0.8, dict(Dmax=-1, chi=100000)),
    ("sq6_chi16", 6, 0.8, dict(Dmax=-1, chi=16)),
    ("sq5_cutbond", 5, 0.8, dict(Dmax=1000, chi=100000, cut_bond=True)),
    ("sq6_d4", 6, 1.0, dict(Dmax=4, chi=16)),
    ("sq8_d8", 8, 0.8, dict(Dmax=8, chi=32)),
    ("sq8_d16_norm2", 8, 1.5, dict(Dmax=16, chi=64, norm_method=2)),
    ("sq8_select2_noreverse", 8, 1.0, dict(Dmax=8, chi=32, select=2, reverse=False)),
]


@pytest.mark.parametrize("name,L,beta,kw", CASES, ids=[c[0] for c in CASES])
def test_against_central_differences(host, name, L, beta, kw):
    r = np.random.default_rng(zlib.crc32(name.encode()) % 1000)
    e = X.square_edges(L)
    n = L * L
    w, h = r.normal(size=len(e)), r.normal(0, 0.2, n)
    st, lz, dw, dh = grad(host, n, e, w, h, beta, **kw)
    assert st == 0
    # these configurations contract without loss: the lnZ is the exact one
    assert abs(lz - X.square_transfer_lnZ(L, L, e, w, h, beta)) / n < 1e-12
    assert fd_check(host, n, e, w, h, beta, dw, dh, **kw) < 1e-8


def test_gradient_run_matches_plain_run(host):
    """The taped contraction computes the same lnZ as the plain engine."""
    from test_hostcheck_engine import run_ising
    r = np.random.default_rng(2)
    e = X.square_edges(8)
    w, h = r.normal(size=len(e)), r.normal(0, 0.1, 64)
    st0, res, _ = run_ising(host, 64, e, w, h, 1.2, Dmax=8, chi=32)
    st1, lz, _, _ = grad(host, 64, e, w, h, 1.2, Dmax=8, chi=32)
    assert st0 == 0 and st1 == 0
    assert lz == res.lnZ


CKPT_CASES = [
    ("sq7_d8", "square", 7, dict(Dmax=8, chi=16)),
    ("sq7_select0_norm2_noreverse", "square", 7, dict(Dmax=8, chi=16, select=0, norm_method=2, reverse=False)),
    ("sq7_select2_norm0_plain_svd", "square", 7, dict(Dmax=8, chi=16, select=2, norm_method=0, svdopt=False,
                                                     swapopt=False)),
    ("sq7_cutbond", "square", 7, dict(Dmax=4, chi=8, cut_bond=True)),
    ("rrg40_d16", "rrg", 40, dict(Dmax=16, chi=32)),
    ("sq4_exact", "square", 4, dict(Dmax=-1, chi=10000)),
]


@pytest.mark.parametrize("name,graph,size,kw", CKPT_CASES, ids=[c[0] for c in CKPT_CASES])
def test_checkpointed_gradients_bit_identical(host, name, graph, size, kw):
    """ckpt_interval K > 0 (segments of K steps recomputed in the backward
    pass from packed checkpoints) gives the whole-tape lnZ and gradients bit
    for bit, for segment lengths that do and do not divide the step count."""
    r = np.random.default_rng(zlib.crc32(name.encode()) % 1000)
    if graph == "square":
        e, n = X.square_edges(size), size * size
    else:
        e, n = X.random_regular_graph(size, 3, r), size
    w, h = r.normal(size=len(e)), r.normal(0, 0.2, n)
    st0, lz0, dw0, dh0 = grad(host, n, e, w, h, 0.7, **kw)
    assert st0 == 0
    for K in (1, 5, 16, 1000):
        st, lz, dw, dh = grad(host, n, e, w, h, 0.7, ckpt_interval=K, **kw)
        assert st == 0
        assert lz == lz0
        np.testing.assert_array_equal(dw, dw0)
        np.testing.assert_array_equal(dh, dh0)


def test_checkpointed_run_fits_where_the_whole_tape_does_not(host):
    """20 x 20 lattice (399 steps): in a 16 MiB arena the whole tape runs out
    of memory, while checkpoints every 64 steps fit and give the gradients of
    the whole-tape run made in a larger arena."""
    r = np.random.default_rng(20)
    e = X.square_edges(20)
    w, h = r.normal(size=len(e)), r.normal(0, 0.2, 400)
    kw = dict(Dmax=4, chi=8)
    st, _, _, _ = grad(host, 400, e, w, h, 0.8, arena=16 << 20, **kw)
    assert st == L.CATN_ENOMEM
    st0, lz0, dw0, dh0 = grad(host, 400, e, w, h, 0.8, arena=64 << 20, **kw)
    st, lz, dw, dh = grad(host, 400, e, w, h, 0.8, arena=16 << 20, ckpt_interval=64, **kw)
    assert st0 == 0 and st == 0
    assert lz == lz0
    np.testing.assert_array_equal(dw, dw0)
    np.testing.assert_array_equal(dh, dh0)


def test_compress_is_rejected(host):
    e = X.square_edges(3)
    st, _, _, _ = grad(host, 9, e, np.ones(len(e)), np.zeros(9), 0.5, Dmax=4, chi=8, compress=True)
    assert st == L.CATN_EINVAL


def test_gradient_memory_safety_asan():
    """The gradient path through the ASan/UBSan build, in a fresh process."""
    so = hostbuild.build(asan=True)
    libasan = subprocess.run(["gcc", "-print-file-name=libasan.so"], capture_output=True, text=True).stdout.strip()
    libubsan = subprocess.run(["gcc", "-print-file-name=libubsan.so"], capture_output=True, text=True).stdout.strip()
    code = f"""
import sys, ctypes as ct, numpy as np
sys.path.insert(0, {os.path.dirname(HERE)!r})
import __graft_entry__; __graft_entry__.load_package()
sys.path.insert(0, {HERE!r})
import test_adjoint_host as T
from oracle import exact as X
lib = ct.CDLL({so!r})
r = np.random.default_rng(3)
for L, kw in [(5, dict(Dmax=4, chi=16)), (5, dict(Dmax=1000, chi=100000, cut_bond=True)), (4, dict(Dmax=-1, chi=100, norm_method=2)),
              (5, dict(Dmax=4, chi=16, ckpt_interval=3))]:
    e = X.square_edges(L)
    st, lz, dw, dh = T.grad(lib, L*L, e, r.normal(size=len(e)), r.normal(0, .1, L*L), 1.0, **kw)
    assert st == 0, st
print("asan-ok")
"""
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1", UBSAN_OPTIONS="halt_on_error=1",
               LD_PRELOAD=f"{libasan}:{libubsan}")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=600)
    assert "asan-ok" in out.stdout, out.stderr[-3000:]
