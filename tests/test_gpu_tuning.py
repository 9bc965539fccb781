"""The process-wide tuning table (catn_tuning_set) moves work between CTAs
only: with the smallest sharing thresholds every SVD and Householder step in
global memory that may be shared is published to helper CTAs, and the
results must be those of the built-in table.  An SVD held in one CTA's shared
memory is never published (its address means nothing to another CTA), which
these thresholds reach: a Jacobi factor of 32 columns fits in shared memory.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SMALLEST = dict(helper_ctas=4, grad_helper_ctas=4, shared_jacobi_min_n=2, shared_house_min=1)


@pytest.fixture
def tuning():
    from catn_b200 import tune
    saved = tune.get()
    yield tune
    tune.apply(saved)


def _batch_lnZ(catn, insts, **kw):
    b = catn.IsingBatch(insts, **kw)
    b.run()
    return np.array(b.lnZ())


def test_batch_results_do_not_depend_on_sharing(catn, tuning):
    from catn_b200 import graphs
    insts = graphs.spinglass_batch(24, 7, sizes=(6, 8, 10))
    ref = _batch_lnZ(catn, insts, Dmax=32, chi=128)
    tuning.apply(SMALLEST)
    got = _batch_lnZ(catn, insts, Dmax=32, chi=128)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)


def test_single_network_results_do_not_depend_on_sharing(catn, tuning):
    """One network per launch: every other CTA helps its shared jobs."""
    from oracle import exact as X
    r = np.random.default_rng(60)
    n = 40
    e = X.random_regular_graph(n, 3, r)
    w, h = r.choice([-1.0, 1.0], size=len(e)), r.normal(0, 0.1, n)
    kw = dict(Dmax=32, chi=128)
    ref = catn.ising_network(n, e, w, h, 1.0, **kw)
    lz_ref = catn.contraction(ref, trace=True)[0]
    tuning.apply(SMALLEST)
    got = catn.ising_network(n, e, w, h, 1.0, **kw)
    lz = catn.contraction(got, trace=True)[0]
    assert lz == pytest.approx(lz_ref, rel=1e-12)
    assert np.array_equal(got.trace, ref.trace)
