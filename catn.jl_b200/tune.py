"""Autotuner for the engine's launch shapes and SVD-route thresholds.

The library keeps one process-wide table (``catn_tuning`` in
include/catn_b200.h): the helper-CTA pools of batch launches, the smallest
SVDs whose Jacobi rounds and Householder steps are shared with helper CTAs,
and the smallest Jacobi factor that takes the block route.  ``tune()``
measures candidate values on the GPU with CUDA events, one family at a time
(the others held at their current values), and returns the winners together
with every measurement; ``apply()`` installs a table in the library and
``load()`` / ``save()`` read and write it as JSON.  The package applies
``tuning_b200.json`` (beside this file) when the library is first loaded,
if that file exists.

The helper and sharing entries change only which CTA does which work
(results are bit-identical for every value); ``block_min_n`` changes which
route computes an SVD and so the rounding of the results, within the
route's stated accuracy.
"""
import ctypes as ct
import json
import os
import time

import numpy as np

from . import _lib as L

TABLE_PATH = L.TUNING_PATH
FIELDS = ("helper_ctas", "grad_helper_ctas", "shared_jacobi_min_n", "block_min_n", "shared_house_min",
          "blocked_qr_min_n", "reserved")


def get():
    """The table in force, as a dict (built-in defaults until changed)."""
    lib = L.load()
    t = L.Tuning()
    L.check(lib, lib.catn_tuning_get(ct.byref(t)))
    return {f: int(getattr(t, f)) for f in FIELDS}


def apply(table):
    """Install the entries of `table` (missing entries keep their value)."""
    lib = L.load()
    cur = get()
    cur.update({k: int(v) for k, v in table.items() if k in FIELDS})
    t = L.Tuning(*[cur[f] for f in FIELDS])
    L.check(lib, lib.catn_tuning_set(ct.byref(t)))
    return cur


def load(path=TABLE_PATH):
    with open(path) as f:
        return json.load(f)


def save(result, path=TABLE_PATH):
    with open(path, "w") as f:
        json.dump(result, f, indent=1, sort_keys=True)


def _cuda_time(fn, repeats):
    import torch
    best = None
    for _ in range(repeats):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        t = a.elapsed_time(b) / 1000.0
        best = t if best is None else min(best, t)
    return best


def tune(batch_instances=512, repeats=3, rrg_n=160, verbose=True):
    """Measure candidates on the current GPU and return {"table": winners,
    "measurements": {...}, "device": name}.  Takes a minute or two."""
    import torch
    from .ising import IsingBatch, ising_network
    from .network import B200, adapt, contraction
    from . import graphs
    meas = {}
    base = get()
    # batch launch: helper pool and the shared-Jacobi threshold
    insts = graphs.spinglass_batch(batch_instances, 2024)
    b = IsingBatch(insts, Dmax=32, chi=128)
    b.upload()
    b.launch()
    b.fetch()
    best = None
    for h in (8, 16, 24):
        for mn in (96, 128):
            apply(dict(base, helper_ctas=h, shared_jacobi_min_n=mn))
            t = _cuda_time(b.launch, repeats)
            meas[f"batch helper_ctas={h} shared_jacobi_min_n={mn}"] = t
            if verbose:
                print(f"  batch  helper_ctas={h:3d} shared_jacobi_min_n={mn:4d}  {1000 * t:8.2f} ms", flush=True)
            if best is None or t < best[0]:
                best = (t, h, mn)
    table = dict(base, helper_ctas=best[1], shared_jacobi_min_n=best[2])
    apply(table)
    # single network on the block route: the route's size threshold, on a
    # random 3-regular glass whose swaps produce Jacobi factors of a few
    # hundred columns
    r = np.random.default_rng(rrg_n)
    e = graphs.random_regular_graph(rrg_n, 3, r)
    w = r.choice([-1.0, 1.0], size=len(e))
    hf = r.normal(0, 0.1, rrg_n)

    def run():
        tn = ising_network(rrg_n, e, w, hf, 1.0, Dmax=32, chi=128, svd_route="block")
        adapt(B200, tn)   # device allocation outside the timed region
        return lambda: contraction(tn)

    run()()   # warm-up (allocation)
    best = None
    for bm in (80, 128, 192, 256, 384):
        apply(dict(table, block_min_n=bm))
        t = _cuda_time(run(), 1)
        meas[f"rrg{rrg_n} block route, block_min_n={bm}"] = t
        if verbose:
            print(f"  rrg{rrg_n} block_min_n={bm:4d}  {t:8.3f} s", flush=True)
        if best is None or t < best[0]:
            best = (t, bm)
    table["block_min_n"] = best[1]
    apply(table)
    return {"table": table, "measurements": meas, "device": torch.cuda.get_device_name(),
            "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}
