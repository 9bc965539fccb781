"""Blocks of destroyed networks and batches are kept by the library and
handed to the next network or batch (pool.cu).  A reused block arrives with
its old contents, so networks contracted in a loop must give the results of
fresh allocations; releasing the cache must give the memory back."""
import gc

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lattice(L, seed):
    from catn_b200.graphs import square_edges
    r = np.random.default_rng(seed)
    e = square_edges(L)
    return L * L, e, r.normal(size=len(e)), r.normal(0, 0.2, L * L)


def test_networks_in_a_loop_reuse_blocks(catn):
    import torch
    catn.release_cached_memory()
    n, e, w, h = _lattice(6, 1)
    first = None
    for k in range(4):
        net = catn.ising_network(n, e, w, h, 0.8, Dmax=16, chi=32)
        catn.adapt(catn.B200, net, trace=True)
        lz = catn.contraction(net, trace=True)[0]
        tr = net.trace.copy()
        if first is None:
            first = (lz, tr)
        else:
            assert lz == first[0] and np.array_equal(tr, first[1])
        # another network in between, of another size, reuses the blocks too
        n2, e2, w2, h2 = _lattice(4 + k, 10 + k)
        catn.contraction(catn.ising_network(n2, e2, w2, h2, 1.0, Dmax=8, chi=16))
        del net
        gc.collect()
    lib = catn.load_library()
    assert lib.catn_cached_bytes(0) > 0 and lib.catn_cached_bytes(1) > 0
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    kept = catn.release_cached_memory()
    assert kept > 0
    assert lib.catn_cached_bytes(0) == 0 and lib.catn_cached_bytes(1) == 0
    assert torch.cuda.mem_get_info()[0] >= free_before + kept // 2


def test_batches_reuse_blocks(catn):
    from catn_b200 import graphs
    insts = graphs.spinglass_batch(12, 3, sizes=(4, 6, 8))
    ref = None
    for _ in range(3):
        b = catn.IsingBatch(insts, Dmax=16, chi=32)
        b.run()
        lz = np.array(b.lnZ())
        if ref is None:
            ref = lz
        else:
            assert np.array_equal(lz, ref)
        del b
        gc.collect()
    catn.release_cached_memory()
