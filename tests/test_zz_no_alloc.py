"""The allocation-free entry point, catn_ising_contract_static, against the
regular path (catn_ising_create + catn_contract).

Some callers cannot call cudaMalloc -- code that runs under a memory pool or
device-memory budget it does not own, or in a loop where allocation latency
is not acceptable.  For them the library contracts one Ising network inside a
fixed device array it holds from load time.  This test calls that entry point
through the C ABI several times in a row (so that each call starts from the
previous call's leftover array contents) and checks every result against the
regular entry point on the same network, with the FP64 parity tolerances of
the other GPU tests.  It lives in its own file, collected last, and needs
nothing from the other tests.
"""
import ctypes as ct

import numpy as np
import pytest

from catn_b200 import _lib as L
from catn_b200 import graphs

pytestmark = pytest.mark.gpu


def _network(L_side, seed):
    rng = np.random.default_rng(seed)
    e = graphs.square_edges(L_side)
    return dict(n=L_side * L_side, edges=np.ascontiguousarray(np.array(e, dtype=np.int32).reshape(-1)),
                m=len(e), w=np.ascontiguousarray(rng.normal(size=len(e))),
                h=np.ascontiguousarray(rng.normal(0, 0.1, L_side * L_side)), beta=float(rng.uniform(0.5, 2.0)))


def _regular(lib, p, d):
    h = ct.c_void_p()
    L.check(lib, lib.catn_ising_create(ct.byref(p), d["n"], d["m"], L.ptr(d["edges"]), L.ptr(d["w"]),
                                       L.ptr(d["h"]), d["beta"], 0, 0, 0, 0, 0, ct.byref(h)))
    res = L.Result()
    try:
        L.check(lib, lib.catn_contract(h, ct.byref(res), None, 0))
    finally:
        lib.catn_net_destroy(h)
    return res


def _static(lib, p, d):
    res = L.Result()
    L.check(lib, lib.catn_ising_contract_static(ct.byref(p), d["n"], d["m"], L.ptr(d["edges"]), L.ptr(d["w"]),
                                                L.ptr(d["h"]), d["beta"], 0, 0, 0, 0, None, ct.byref(res)))
    return res


def test_static_scratch_matches_regular_path_on_consecutive_calls():
    lib = L.load()
    p = L.make_params(Dmax=32, chi=128)
    nets = [_network(8, 1), _network(10, 2), _network(8, 1), _network(12, 3)]
    refs = [_regular(lib, p, d) for d in nets]
    for d, ref in zip(nets, refs):
        got = _static(lib, p, d)
        assert got.status == 0
        assert got.nsteps == ref.nsteps
        assert got.maxdim == ref.maxdim
        assert got.psi == ref.psi
        assert abs(got.lnZ - ref.lnZ) / d["n"] <= 1e-10
        assert abs(got.err - ref.err) <= 1e-12 + 1e-6 * abs(ref.err)


def test_static_scratch_rejects_oversized_network():
    lib = L.load()
    p = L.make_params(Dmax=32, chi=128)
    d = _network(64, 4)   # its pair map alone (4097^2 ints) exceeds the fixed array
    res = L.Result()
    st = lib.catn_ising_contract_static(ct.byref(p), d["n"], d["m"], L.ptr(d["edges"]), L.ptr(d["w"]),
                                        L.ptr(d["h"]), d["beta"], 0, 0, 0, 0, None, ct.byref(res))
    assert st == L.CATN_ENOMEM
    assert "static maximum" in L.last_error(lib)
