"""bench.py's secondary legs run end to end on the CPU against a stand-in
for the package (no device): a Python error in a leg would otherwise only
show on the GPU box, where it would cost the whole bench line.  The numbers
are meaningless here; the keys and the comparisons with the frozen fixtures
are what is checked."""
import json
import os
import sys
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


class _Result:
    def __init__(self):
        self.prof = [1.0] * 24
        self.flops = 1.0
        self.bytes = 1.0
        self.arena_peak = 1 << 20


class _Net:
    def __init__(self, rows, lnZ, n=0, n_edges=0):
        self.result = _Result()
        self.trace = None
        self.maxdim_intermediate = 1
        self._rows, self._lnZ = rows, lnZ
        self.n, self.n_edges = n, n_edges


def _fake(rows, lnZ):
    """A stand-in whose networks report the given trace rows and lnZ."""
    f = types.SimpleNamespace(B200="b200")
    f.ising_network = lambda n, e, w, h, beta, **kw: _Net(rows, lnZ, n, len(e))
    f.TensorNetwork = lambda et, ei, **kw: _Net(rows, lnZ)
    f.adapt = lambda to, net, **kw: net

    def contraction(net, trace=False):
        if trace:
            net.trace = np.array([list(r) + [0] for r in net._rows], dtype=np.int32)
        return net._lnZ, 0.0, 1.0
    f.contraction = contraction
    f.gradient = lambda net, ckpt_interval=None: (lnZ, np.zeros(net.n_edges), np.zeros(net.n))

    class IsingBatch:
        def __init__(self, insts, **kw):
            self.n = len(insts)
            self.slots = 1

        def run(self):
            pass

        def lnZ(self):
            return np.zeros(self.n)
    f.IsingBatch = IsingBatch
    return f


@pytest.fixture(autouse=True)
def _no_oracle_timing(monkeypatch):
    monkeypatch.setattr(bench, "_time_oracle", lambda name: {"s": 0.0, "lnZ": 0.0, "cores": 1, "what": "stub"})


def test_gaussian_lattice_reduced_leg():
    d = json.load(open(os.path.join(GOLDEN, "gaussian10.json")))
    out = bench.c4_reduced_leg(_fake(d["oracle"]["trace"], d["oracle"]["lnZ"]))
    assert out["vs_oracle"]["trace_identical"] and out["vs_oracle"]["abs_dlnZ_per_site"] == 0.0
    assert out["pinning_networks"] == 1 + 2 * d["n"] + 4 * len(d["edges"])
    json.dumps(out)


def test_peps_reduced_leg():
    d = json.load(open(os.path.join(GOLDEN, "peps6.json")))
    import __graft_entry__
    __graft_entry__.load_package()
    out = bench.peps_reduced_leg(_fake(d["oracle"]["trace"], d["oracle"]["lnZ"]))
    assert set(out["forms"]) == {"fp64_scalar", "fp64_block", "split"}
    assert all(f["trace_identical_to_oracle"] for f in out["forms"].values())
    json.dumps(out)


def test_random_regular_leg():
    d = json.load(open(os.path.join(GOLDEN, "rrg200.json")))
    args = types.SimpleNamespace(c2_scalar=False, no_c2_oracle=True)
    out = bench.c2_leg(_fake(d["oracle"][0]["trace"], d["oracle"][0]["lnZ"]), args, 35.0, 1400.0)
    assert set(out["forms"]) == {"fp64_block", "split"}
    assert out["forms"]["fp64_block"]["runs"][0]["trace_identical"]
    json.dumps(out)


def test_full_size_lattice_leg():
    out = bench.c4_full_leg(_fake([], 1.0), L=4, pin_edges=2)
    assert out["pinning_subset_networks"] == 1 + 4 * 2
    json.dumps(out)


def test_a_failing_leg_is_recorded_not_raised():
    out = {}
    bench._secondary(out, "ok", lambda: {"value": 1})

    def boom():
        raise RuntimeError("device lost")
    bench._secondary(out, "bad", boom)
    assert out["ok"] == {"value": 1}
    assert out["bad"] == {"error": "RuntimeError: device lost"}
