"""The frozen fixtures that bench.py compares with are the oracle's output:
regenerate the fast ones on the CPU and compare (the n = 200 random-regular
and the 6x6 PEPS fixtures take tens of seconds of oracle time and are made by
tests/golden/make_golden.py)."""
import json
import os

import numpy as np

from oracle import exact as X
from oracle import ising as OI
from oracle import network as ON

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fnv(vals):
    h = 2166136261
    for v in vals:
        h = ((h ^ (v & 0xffffffff)) * 16777619) & 0xffffffff
    return h - (1 << 32) if h >= (1 << 31) else h


def _rows():
    return [[i, j, int(ri) | (int(rj) << 1), len(d), fnv(d), len(s), fnv(s)] for (i, j, ri, rj, d, s) in ON.TRACE]


def test_gaussian10_fixture_is_the_oracle_output():
    d = json.load(open(os.path.join(HERE, "gaussian10.json")))
    rng = np.random.default_rng(4)
    e = X.square_edges(d["L"])
    assert [list(x) for x in e] == d["edges"]
    assert np.array_equal(rng.normal(size=len(e)), d["weights"])
    assert np.array_equal(rng.normal(0, 0.2, d["n"]), d["fields"])
    ON.TRACE = []
    tn = OI.ising_network(d["n"], d["edges"], d["weights"], d["fields"], d["beta"], **d["params"])
    lnZ, err, psi = ON.contraction(tn)
    rows = _rows()
    ON.TRACE = None
    assert rows == d["oracle"]["trace"]
    assert lnZ == d["oracle"]["lnZ"] and psi == d["oracle"]["psi"]


def test_ferro8_fixture_matches_the_transfer_matrix():
    d = json.load(open(os.path.join(HERE, "config1_ferro8.json")))
    assert abs(d["oracle"]["lnZ"] - d["exact_lnZ"]) / d["n"] < 1e-12
