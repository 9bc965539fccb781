"""The plain GPU form (baseline/plain_gpu_form.py, the PyTorch FP64
one-library-call-per-op restatement that bench.py times beside the engine)
against the oracle, run on the CPU device: same lnZ, error, psi and
maxdim_intermediate on the same networks."""
import os
import sys
import zlib

import numpy as np
import pytest

from oracle import exact as X
from oracle import ising as OI
from oracle import network as ON

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "baseline"))
import plain_gpu_form as PG  # noqa: E402

sys.path.pop(0)

CASES = [
    ("sq6_d8", 6, 1.0, dict(Dmax=8, chi=32)),
    ("sq8_d32", 8, 1.2, dict(Dmax=32, chi=128)),
    ("sq6_select0", 6, 0.9, dict(Dmax=16, chi=64, select=0)),
    ("sq6_select2", 6, 0.9, dict(Dmax=16, chi=64, select=2)),
    ("sq6_compress", 6, 1.0, dict(Dmax=4, chi=16, compress=True)),
    ("sq5_exact", 5, 0.7, dict(Dmax=-1, chi=100000)),
]


@pytest.mark.parametrize("name,L,beta,kw", CASES, ids=[c[0] for c in CASES])
def test_plain_form_matches_oracle(name, L, beta, kw):
    r = np.random.default_rng(zlib.crc32(name.encode()) % 1000)
    e = X.square_edges(L)
    w, h = r.normal(size=len(e)), r.normal(0, 0.1, L * L)
    tn = OI.ising_network(L * L, e, w, h, beta, **kw)
    lz, err, psi = ON.contraction(tn)
    pn = PG.ising_network(L * L, e, w, h, beta, device="cpu", **kw)
    plz, perr, ppsi = PG.contraction(pn)
    assert abs(plz - lz) / (L * L) < 1e-12
    assert abs(perr - err) <= 1e-12 + 1e-6 * abs(err)
    assert ppsi == psi
    assert pn.maxdim == tn.maxdim_intermediate
    if kw["Dmax"] < 0:
        assert plz == pytest.approx(X.square_transfer_lnZ(L, L, e, w, h, beta), rel=1e-9)


def test_plain_form_pinned_random_regular():
    r = np.random.default_rng(8)
    e = X.random_regular_graph(20, 3, r)
    w, h = r.choice([-1.0, 1.0], size=len(e)), r.normal(0, 0.1, 20)
    for pins in [dict(), dict(pos1=3, val1=1), dict(pos1=2, val1=2, pos2=7, val2=1)]:
        lz, _, _ = ON.contraction(OI.ising_network(20, e, w, h, 1.0, Dmax=8, chi=32, **pins))
        plz, _, _ = PG.contraction(PG.ising_network(20, e, w, h, 1.0, device="cpu", Dmax=8, chi=32, **pins))
        assert abs(plz - lz) / 20 < 1e-12
