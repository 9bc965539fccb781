"""The device engine's source compiled for the host (team of one thread,
tests/hostcheck) against the oracle: integer trace bit-exact, lnZ within
1e-12 per spin, plus one AddressSanitizer/UBSan run in a subprocess.

This checks the engine's control logic and memory safety on the CPU; the
GPU parity tests (test_gpu_parity.py) check the CUDA build itself.
"""
import ctypes as ct
import os
import subprocess
import zlib
import sys

import numpy as np
import pytest

from oracle import exact as X
from oracle import ising as OI
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


def oracle_rows(tr):
    return [(i, j, int(ri) | (int(rj) << 1), len(d), fnv(d), len(s), fnv(s)) for (i, j, ri, rj, d, s) in tr]


@pytest.fixture(scope="module")
def host():
    lib = ct.CDLL(hostbuild.build())
    return lib


def run_ising(lib, n, e, w, h, beta, pins=(0, 0, 0, 0), **kw):
    p = L.make_params(**kw)
    E = np.ascontiguousarray(np.array(e, dtype=np.int32).reshape(-1)) if len(e) else np.zeros(2, np.int32)
    W = np.ascontiguousarray(np.array(w, dtype=np.float64)) if len(w) else np.zeros(1)
    H = np.ascontiguousarray(np.array(h, dtype=np.float64))
    cap = 4 * len(e) + 16
    tr = np.zeros(8 * cap, dtype=np.int32)
    res = L.Result()
    st = lib.catn_hostcheck_ising(ct.byref(p), ct.c_int(n), ct.c_int(len(e)), L.ptr(E), L.ptr(W), L.ptr(H),
                                  ct.c_double(beta), *[ct.c_int(x) for x in pins], ct.c_longlong(1 << 30),
                                  ct.byref(res), L.ptr(tr), ct.c_int(cap))
    rows = [tuple(int(x) for x in tr[8 * s:8 * s + 7]) for s in range(min(res.nsteps, cap))]
    return st, res, rows


def oracle_ising(n, e, w, h, beta, pins=(0, 0, 0, 0), **kw):
    ON.TRACE = []
    tn = OI.ising_network(n, e, w, h, beta, pos1=pins[0], val1=pins[1], pos2=pins[2], val2=pins[3], **kw)
    out = ON.contraction(tn)
    tr = ON.TRACE
    ON.TRACE = None
    return out, oracle_rows(tr), tn


CASES = [
    ("square4_exact", 4, 0.7, dict(Dmax=-1, chi=100000)),
    ("square6_d32", 6, 1.0, dict(Dmax=32, chi=128)),
    ("square8_d8", 8, 1.3, dict(Dmax=8, chi=32)),
    ("square8_d4_compress", 8, 1.0, dict(Dmax=4, chi=16, compress=True)),
    ("square8_d4_compress_plain", 8, 1.0, dict(Dmax=4, chi=16, compress=True, svdopt=False)),
    ("square6_select0", 6, 0.9, dict(Dmax=16, chi=64, select=0)),
    ("square6_select2", 6, 0.9, dict(Dmax=16, chi=64, select=2)),
    ("square6_noreverse", 6, 0.9, dict(Dmax=16, chi=64, reverse=False)),
    ("square6_cutbond", 6, 0.9, dict(Dmax=16, chi=64, cut_bond=True)),
    ("square6_norm2", 6, 0.9, dict(Dmax=16, chi=64, norm_method=2)),
    ("square10_d32", 10, 1.0, dict(Dmax=32, chi=128)),
]


@pytest.mark.parametrize("name,L,beta,kw", CASES, ids=[c[0] for c in CASES])
def test_square_spin_glass_trace_and_lnZ(host, name, L, beta, kw):
    r = np.random.default_rng(zlib.crc32(name.encode()) % 1000)
    e = X.square_edges(L)
    w, h = r.normal(size=len(e)), r.normal(0, 0.1, L * L)
    st, res, rows = run_ising(host, L * L, e, w, h, beta, **kw)
    (lz, err, psi), orows, tn = oracle_ising(L * L, e, w, h, beta, **kw)
    assert st == 0 and res.status == 0
    assert rows == orows
    assert abs(res.lnZ - lz) / (L * L) < 1e-12
    assert res.maxdim == tn.maxdim_intermediate
    assert res.psi == psi
    assert abs(res.err - err) <= 1e-12 + 1e-6 * abs(err)


def test_random_regular_graph(host):
    r = np.random.default_rng(5)
    e = X.random_regular_graph(24, 3, r)
    w, h = r.choice([-1.0, 1.0], size=len(e)), r.normal(0, 0.1, 24)
    kw = dict(Dmax=8, chi=32)
    st, res, rows = run_ising(host, 24, e, w, h, 1.0, **kw)
    (lz, err, psi), orows, _ = oracle_ising(24, e, w, h, 1.0, **kw)
    assert st == 0 and rows == orows and abs(res.lnZ - lz) / 24 < 1e-12


def test_pinned_and_isolated(host):
    e, w, h = [(1, 2), (2, 3), (3, 1)], [0.4, 0.6, -0.3], [0.1, -0.2, 0.05]
    for pins in [(1, 1, 0, 0), (2, 2, 0, 0), (1, 2, 3, 1)]:
        st, res, rows = run_ising(host, 3, e, w, h, 0.35, pins=pins, Dmax=-1, chi=10000)
        (lz, _, _), orows, _ = oracle_ising(3, e, w, h, 0.35, pins=pins, Dmax=-1, chi=10000)
        assert st == 0 and rows == orows and res.lnZ == pytest.approx(lz, abs=1e-13)
    st, res, _ = run_ising(host, 3, [(1, 2)], [0.5], [0.2, -0.4, 0.3], 0.5, Dmax=-1, chi=100)
    (lz, _, _), _, _ = oracle_ising(3, [(1, 2)], [0.5], [0.2, -0.4, 0.3], 0.5, Dmax=-1, chi=100)
    assert st == 0 and res.lnZ == pytest.approx(lz, abs=1e-13)


def run_dense(lib, ts, ixs, **kw):
    from catn_b200.network import TensorNetwork
    tn = TensorNetwork(ts, ixs, **kw)   # label resolution only (no device work)
    p = L.make_params(**tn.params)
    ndims = np.array([t.ndim for t in tn.tensors], dtype=np.int32)
    dims = np.array([d for t in tn.tensors for d in t.shape] or [0], dtype=np.int64)
    data = np.ascontiguousarray(np.concatenate([np.ravel(t, order="F") for t in tn.tensors]))
    nbrs = np.array([v for ix in tn.neighbors for v in ix], dtype=np.int32)
    res = L.Result()
    tr = np.zeros(8 * 256, dtype=np.int32)
    st = lib.catn_hostcheck_dense(ct.byref(p), ct.c_int(tn.n), L.ptr(ndims), L.ptr(dims), L.ptr(data), L.ptr(nbrs),
                                  ct.c_longlong(1 << 28), ct.byref(res), L.ptr(tr), ct.c_int(256))
    return st, res


@pytest.mark.parametrize("sel", [0, 1, 2])
@pytest.mark.parametrize("comp", [False, True])
def test_dense_exact_mode(host, sel, comp):
    r = np.random.default_rng(40 + sel)
    nets = [
        ([r.normal(size=(3, 4)), r.normal(size=(4, 5)), r.normal(size=(5, 3))], [["a", "b"], ["b", "c"], ["c", "a"]]),
        ([r.normal(size=(2, 3, 4)), r.normal(size=2), r.normal(size=3), r.normal(size=4)],
         [["a", "b", "c"], ["a"], ["b"], ["c"]]),
        ([r.normal(size=(2, 3)), r.normal(size=(3, 2)), r.normal(size=(2, 3)), r.normal(size=(3, 2))],
         [["a", "b"], ["b", "c"], ["c", "d"], ["d", "a"]]),
    ]
    for ts, ixs in nets:
        ref = float(X.exact_contract(ts, ixs))
        st, res = run_dense(host, ts, ixs, Dmax=-1, chi=10000, select=sel, compress=comp)
        assert st == 0
        assert np.exp(res.lnZ) * res.psi == pytest.approx(ref, rel=1e-10)


def test_engine_memory_safety_asan():
    """Run a few networks through the ASan/UBSan build in a fresh process."""
    so = hostbuild.build(asan=True)
    libasan = subprocess.run(["gcc", "-print-file-name=libasan.so"], capture_output=True, text=True).stdout.strip()
    libubsan = subprocess.run(["gcc", "-print-file-name=libubsan.so"], capture_output=True, text=True).stdout.strip()
    code = f"""
import sys, ctypes as ct, numpy as np
sys.path.insert(0, {os.path.dirname(HERE)!r})
import __graft_entry__; __graft_entry__.load_package()
sys.path.insert(0, {HERE!r})
import test_hostcheck_engine as T
from oracle import exact as X
lib = ct.CDLL({so!r})
r = np.random.default_rng(3)
for L, kw in [(6, dict(Dmax=8, chi=32)), (6, dict(Dmax=4, chi=16, compress=True)), (5, dict(Dmax=-1, chi=10000, select=2))]:
    e = X.square_edges(L)
    st, res, rows = T.run_ising(lib, L*L, e, r.normal(size=len(e)), r.normal(0, .1, L*L), 1.0, **kw)
    assert st == 0, st
# every SVD on the global path, the block route and the blocked QR through the
# shared-job protocol (the item workspaces at their smallest)
import os
os.environ.update(CATN_HOSTCHECK_SWS="0", CATN_HOSTCHECK_BLOCK_MIN="16", CATN_HOSTCHECK_JOB="1",
                  CATN_HOSTCHECK_BLOCKED_QR_MIN="16")
e = X.square_edges(10)
st, res, rows = T.run_ising(lib, 100, e, r.normal(size=len(e)), r.normal(0, .1, 100), 1.3, Dmax=16, chi=96,
                            svd_route="block")
assert st == 0, st
for k in ("CATN_HOSTCHECK_SWS", "CATN_HOSTCHECK_BLOCK_MIN", "CATN_HOSTCHECK_JOB", "CATN_HOSTCHECK_BLOCKED_QR_MIN"):
    del os.environ[k]
# cut_bondim! / cut_bondim_opt! replayed before a contraction
import test_cut_bondim as TC
ts, ixs = TC.grid(3, 4, 11)
st, res, _ = TC.host_run(lib, ts, ixs, TC.CUTS, 0, **TC.KW)
assert st == 0, st
print("asan-ok")
"""
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1", UBSAN_OPTIONS="halt_on_error=1",
               LD_PRELOAD=f"{libasan}:{libubsan}")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=600)
    assert "asan-ok" in out.stdout, out.stderr[-3000:]


@pytest.mark.parametrize("name,L,beta,kw", CASES[:6], ids=[c[0] for c in CASES[:6]])
def test_large_svd_path_everywhere(host, name, L, beta, kw, monkeypatch):
    """Every SVD through the global-memory path with rank-revealing pivoted QR
    (the shared-memory workspace disabled): same trace, same lnZ."""
    monkeypatch.setenv("CATN_HOSTCHECK_SWS", "0")
    r = np.random.default_rng(zlib.crc32(name.encode()) % 1000)
    e = X.square_edges(L)
    w, h = r.normal(size=len(e)), r.normal(0, 0.1, L * L)
    st, res, rows = run_ising(host, L * L, e, w, h, beta, **kw)
    (lz, err, psi), orows, tn = oracle_ising(L * L, e, w, h, beta, **kw)
    assert st == 0 and rows == orows
    assert abs(res.lnZ - lz) / (L * L) < 1e-12
    assert abs(res.err - err) <= 1e-12 + 1e-6 * abs(err)


@pytest.mark.parametrize("name,L,beta,kw", CASES[:4], ids=[c[0] for c in CASES[:4]])
def test_shared_jacobi_protocol(host, name, L, beta, kw, monkeypatch):
    """Every SVD through the global path with its Jacobi sweeps run through the
    shared-job protocol that idle CTAs join on the GPU (here the team claims
    every pair itself): same trace, same lnZ."""
    monkeypatch.setenv("CATN_HOSTCHECK_SWS", "0")
    monkeypatch.setenv("CATN_HOSTCHECK_JOB", "1")
    r = np.random.default_rng(zlib.crc32(name.encode()) % 1000)
    e = X.square_edges(L)
    w, h = r.normal(size=len(e)), r.normal(0, 0.1, L * L)
    st, res, rows = run_ising(host, L * L, e, w, h, beta, **kw)
    (lz, err, psi), orows, tn = oracle_ising(L * L, e, w, h, beta, **kw)
    assert st == 0 and rows == orows
    assert abs(res.lnZ - lz) / (L * L) < 1e-12


def test_shared_wait_timeout_reports_etimeout(host, monkeypatch):
    """The owner's bounded wait for claimed items of a shared round
    (linalg.cuh job_round) runs out: the timeout build of the harness
    publishes every round with one claim that is never reported done (a
    helper that stopped) and polls at most 2000 times.  The instance must end
    with CATN_ETIMEOUT instead of waiting, and a following network on the
    regular build must still complete."""
    stall = ct.CDLL(hostbuild.build(stall=True))
    r = np.random.default_rng(3)
    L_ = 8
    e = X.square_edges(L_)
    w, h = r.normal(size=len(e)), r.normal(0, 0.1, L_ * L_)
    kw = dict(Dmax=8, chi=32)
    # without the shared path the timeout build contracts normally
    st, res, _ = run_ising(stall, L_ * L_, e, w, h, 1.0, **kw)
    assert st == 0 and res.status == 0
    # every large SVD through the shared protocol: the first round times out
    monkeypatch.setenv("CATN_HOSTCHECK_JOB", "1")
    monkeypatch.setenv("CATN_HOSTCHECK_SWS", "0")
    st, res, _ = run_ising(stall, L_ * L_, e, w, h, 1.0, **kw)
    assert st == L.CATN_ETIMEOUT and res.status == L.CATN_ETIMEOUT
    # the regular build on the same shared path completes and matches the oracle
    st, res, rows = run_ising(host, L_ * L_, e, w, h, 1.0, **kw)
    (lz, _, _), orows, _ = oracle_ising(L_ * L_, e, w, h, 1.0, **kw)
    assert st == 0 and res.status == 0 and rows == orows
    assert abs(res.lnZ - lz) / (L_ * L_) < 1e-12


BLOCK_CASES = [
    ("block_l12_d32", 12, 1.5, dict(Dmax=32, chi=128), False),
    ("block_l14_d32_shared", 14, 1.5, dict(Dmax=32, chi=128), True),
    ("block_l12_d16_select0", 12, 1.3, dict(Dmax=16, chi=96, select=0), True),
]


def _lattice(name, L_):
    r = np.random.default_rng(zlib.crc32(name.encode()) % 1000)
    e = X.square_edges(L_)
    return e, r.normal(size=len(e)), r.normal(0, 0.1, L_ * L_)


@pytest.mark.parametrize("name,L_,beta,kw,shared", BLOCK_CASES, ids=[c[0] for c in BLOCK_CASES])
def test_block_route_matches_oracle(host, monkeypatch, name, L_, beta, kw, shared):
    """Every SVD on the global path (workspace capacity 0), Jacobi factors of
    >= 16 columns on the block route (svd_route = 2), alone or through the
    shared-job protocol: the integer trace identical to the oracle's, lnZ
    within 1e-12 per spin (the route's singular values carry absolute error
    ~ eps sigma_1, like LAPACK's), and a different rounding history than the
    scalar route (the block route was taken)."""
    monkeypatch.setenv("CATN_HOSTCHECK_SWS", "0")
    monkeypatch.setenv("CATN_HOSTCHECK_BLOCK_MIN", "16")
    if shared:
        monkeypatch.setenv("CATN_HOSTCHECK_JOB", "1")
        # the blocked, norm-sorted QR in place of the pivoted one
        monkeypatch.setenv("CATN_HOSTCHECK_BLOCKED_QR_MIN", "16")
    e, w, h = _lattice(name, L_)
    st, res, rows = run_ising(host, L_ * L_, e, w, h, beta, svd_route="block", **kw)
    (lz, err, psi), orows, tn = oracle_ising(L_ * L_, e, w, h, beta, **kw)
    assert st == 0 and res.status == 0
    assert rows == orows
    assert abs(res.lnZ - lz) / (L_ * L_) < 1e-12
    assert res.maxdim == tn.maxdim_intermediate
    assert abs(res.err - err) <= 1e-10 + 1e-8 * abs(err)
    st, res_s, _ = run_ising(host, L_ * L_, e, w, h, beta, svd_route="scalar", **kw)
    assert st == 0 and (res_s.lnZ, res_s.err) != (res.lnZ, res.err)


def test_block_route_random_regular_graph(host, monkeypatch):
    """A random 3-regular +-1 glass (n = 110, Dmax 32, chi 128) whose swaps
    reach 512-column factors, through the shared-job protocol on the
    default block threshold's side of the route."""
    monkeypatch.setenv("CATN_HOSTCHECK_SWS", "0")
    monkeypatch.setenv("CATN_HOSTCHECK_BLOCK_MIN", "80")
    monkeypatch.setenv("CATN_HOSTCHECK_BLOCKED_QR_MIN", "80")
    monkeypatch.setenv("CATN_HOSTCHECK_JOB", "1")
    r = np.random.default_rng(110)
    e = X.random_regular_graph(110, 3, r)
    w, h = r.choice([-1.0, 1.0], size=len(e)), r.normal(0, 0.1, 110)
    kw = dict(Dmax=32, chi=128)
    st, res, rows = run_ising(host, 110, e, w, h, 1.0, svd_route="block", **kw)
    (lz, err, psi), orows, _ = oracle_ising(110, e, w, h, 1.0, **kw)
    assert st == 0 and rows == orows
    assert abs(res.lnZ - lz) / 110 < 1e-12
    assert abs(res.err - err) <= 1e-10 + 1e-8 * abs(err)
