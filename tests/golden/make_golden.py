"""Generate tests/golden/*.json from the oracle and the exact checkers.

    python tests/golden/make_golden.py

Fixtures (seeded synthetic inputs with the workload shapes):
  config1_ferro8.json    8x8 open ferromagnet, beta 0.44, Dmax 20, chi 200:
                         exact lnZ (row transfer matrix), oracle lnZ/err/trace
  spinglass_sample.json  12 instances of the batched spin-glass workload
                         (L in {8..16}, J~N(0,1), h~N(0,0.01), beta~U[0.5,2],
                         Dmax 32, chi 128): oracle lnZ/err/steps/trace rows,
                         exact lnZ for L <= 12
  rrg_sample.json        n=24 random 3-regular +-1 spin glass, beta in
                         {0.5,1,1.5}, Dmax 8, chi 32 (small stand-in for the
                         n=200 configuration): oracle lnZ/err/trace
  rrg200.json            the n=200 random 3-regular +-1 spin glass itself
                         (300 edges, h~N(0,0.01), beta in {0.5,1,1.5}, Dmax 32,
                         chi 128): oracle lnZ/err/psi/maxdim/trace (about 35 s
                         of oracle time per beta, hence frozen here)

  gaussian10.json        the 32x32 Gaussian configuration reduced to L = 10
                         (J~N(0,1), h~N(0,0.2^2), beta 1, Dmax 48, chi 256,
                         seed 4, the bench's reduced leg): inputs and oracle
                         lnZ/err/psi/maxdim/trace
  peps6.json             the 16x16 PEPS norm configuration reduced to a 6x6
                         double layer (d 2, D 3, Dmax 64, chi 128, seed 506,
                         graphs.peps_double_layer): oracle lnZ/err/psi/trace

    python tests/golden/make_golden.py [name ...]   # regenerate only these
The trace row format is the device's (see include/catn_b200.h).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import exact as X  # noqa: E402
from oracle import ising as OI  # noqa: E402
from oracle import network as ON  # noqa: E402


def fnv(vals):
    h = 2166136261
    for v in vals:
        h = ((h ^ (v & 0xffffffff)) * 16777619) & 0xffffffff
    return h - (1 << 32) if h >= (1 << 31) else h


def run(n, e, w, h, beta, **kw):
    ON.TRACE = []
    tn = OI.ising_network(n, e, w, h, beta, **kw)
    lnZ, err, psi = ON.contraction(tn)
    rows = [[i, j, int(ri) | (int(rj) << 1), len(d), fnv(d), len(s), fnv(s)] for (i, j, ri, rj, d, s) in ON.TRACE]
    ON.TRACE = None
    return dict(lnZ=lnZ, err=err, psi=psi, maxdim=tn.maxdim_intermediate, steps=len(rows), trace=rows)


def spinglass(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        L = int(rng.choice([8, 10, 12, 14, 16]))
        e = X.square_edges(L)
        out.append(dict(L=L, n=L * L, edges=e, weights=rng.normal(size=len(e)).tolist(),
                        fields=rng.normal(0, 0.1, L * L).tolist(), beta=float(rng.uniform(0.5, 2.0))))
    return out


def _trace_rows():
    return [[i, j, int(ri) | (int(rj) << 1), len(d), fnv(d), len(s), fnv(s)] for (i, j, ri, rj, d, s) in ON.TRACE]


def gaussian10():
    rng = np.random.default_rng(4)
    L = 10
    e = X.square_edges(L)
    w = rng.normal(size=len(e)).tolist()
    h = rng.normal(0, 0.2, L * L).tolist()
    d = dict(L=L, n=L * L, edges=e, weights=w, fields=h, beta=1.0, params=dict(Dmax=48, chi=256, cutoff=1e-15))
    d["oracle"] = run(L * L, e, w, h, 1.0, Dmax=48, chi=256)
    json.dump(d, open(os.path.join(HERE, "gaussian10.json"), "w"))


def peps6():
    import __graft_entry__
    __graft_entry__.load_package()
    from catn_b200 import graphs
    d = dict(L=6, D=3, d=2, seed=506, params=dict(Dmax=64, chi=128, cutoff=1e-15))
    _, _, et, ei = graphs.peps_double_layer(6, 3, 2, np.random.default_rng(506))
    ON.TRACE = []
    tn = ON.TensorNetwork.from_tensors(et, ei, Dmax=64, chi=128)
    lnZ, err, psi = ON.contraction(tn)
    rows = _trace_rows()
    ON.TRACE = None
    d["oracle"] = dict(lnZ=lnZ, err=err, psi=psi, maxdim=tn.maxdim_intermediate, steps=len(rows), trace=rows)
    json.dump(d, open(os.path.join(HERE, "peps6.json"), "w"))


def rrg200():
    rng = np.random.default_rng(200)
    e = X.random_regular_graph(200, 3, rng)
    w = rng.choice([-1.0, 1.0], size=len(e)).tolist()
    h = rng.normal(0, 0.1, 200).tolist()
    d = dict(n=200, edges=e, weights=w, fields=h, params=dict(Dmax=32, chi=128, cutoff=1e-15), betas=[0.5, 1.0, 1.5])
    d["oracle"] = [run(200, e, w, h, b, Dmax=32, chi=128) for b in d["betas"]]
    json.dump(d, open(os.path.join(HERE, "rrg200.json"), "w"))


def main():
    only = set(sys.argv[1:])
    if only:
        if "rrg200" in only:
            rrg200()
        if "gaussian10" in only:
            gaussian10()
        if "peps6" in only:
            peps6()
        print("golden fixtures written:", " ".join(sorted(only)))
        return
    e = X.square_edges(8)
    w, h = [1.0] * len(e), [0.0] * 64
    c1 = dict(n=64, edges=e, weights=w, fields=h, beta=0.44, params=dict(Dmax=20, chi=200, cutoff=1e-15))
    c1["oracle"] = run(64, e, w, h, 0.44, Dmax=20, chi=200)
    c1["exact_lnZ"] = X.square_transfer_lnZ(8, 8, e, w, h, 0.44)
    json.dump(c1, open(os.path.join(HERE, "config1_ferro8.json"), "w"))

    insts = spinglass(12, 77)
    for d in insts:
        d["oracle"] = run(d["n"], d["edges"], d["weights"], d["fields"], d["beta"], Dmax=32, chi=128)
        if d["L"] <= 12:
            d["exact_lnZ"] = X.square_transfer_lnZ(d["L"], d["L"], d["edges"], d["weights"], d["fields"], d["beta"])
    json.dump(dict(params=dict(Dmax=32, chi=128, cutoff=1e-15), instances=insts),
              open(os.path.join(HERE, "spinglass_sample.json"), "w"))

    rng = np.random.default_rng(24)
    e = X.random_regular_graph(24, 3, rng)
    w = rng.choice([-1.0, 1.0], size=len(e)).tolist()
    h = rng.normal(0, 0.1, 24).tolist()
    rr = dict(n=24, edges=e, weights=w, fields=h, params=dict(Dmax=8, chi=32, cutoff=1e-15), betas=[0.5, 1.0, 1.5])
    rr["oracle"] = [run(24, e, w, h, b, Dmax=8, chi=32) for b in rr["betas"]]
    rr["exact_lnZ"] = [X.brute_lnZ(24, e, w, h, b) for b in rr["betas"]]
    json.dump(rr, open(os.path.join(HERE, "rrg_sample.json"), "w"))
    rrg200()
    print("golden fixtures written")


if __name__ == "__main__":
    main()
