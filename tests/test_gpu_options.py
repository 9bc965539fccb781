"""GPU trace parity for every option of ``contraction!`` on Ising lattices.

The reference's own test matrix sweeps ``select``, ``reverse``, ``compress``
and the bond-cut options (test/test_contraction.jl:69-88); its MPS-node tests
cover ``norm_method``, ``svdopt`` and ``swapopt`` (test/test_mps_node.jl).
Each case here runs one truncated spin glass through the C ABI on the GPU and
holds it to the oracle: the per-step integer trace (edge, reverse flags,
duplicate list, phys-dim sequence) identical, |dlnZ|/n <= 1e-10, psi and
maxdim_intermediate equal, and err within 1e-6 relative.
"""
import zlib

import numpy as np
import pytest

from oracle import exact as X
from oracle import ising as OI
from oracle import network as ON

pytestmark = pytest.mark.gpu


def fnv(vals):
    h = 2166136261
    for v in vals:
        h = ((h ^ (v & 0xffffffff)) * 16777619) & 0xffffffff
    return h - (1 << 32) if h >= (1 << 31) else h


def oracle_rows(tr):
    return [(i, j, int(ri) | (int(rj) << 1), len(d), fnv(d), len(s), fnv(s)) for (i, j, ri, rj, d, s) in tr]


CASES = [
    ("select0", 6, 0.9, dict(Dmax=16, chi=64, select=0)),
    ("select2", 6, 0.9, dict(Dmax=16, chi=64, select=2)),
    ("select0_l8", 8, 1.2, dict(Dmax=8, chi=32, select=0)),
    ("select2_l8", 8, 1.2, dict(Dmax=8, chi=32, select=2)),
    ("noreverse", 6, 0.9, dict(Dmax=16, chi=64, reverse=False)),
    ("noreverse_l8", 8, 1.2, dict(Dmax=8, chi=32, reverse=False)),
    ("norm0", 6, 0.9, dict(Dmax=16, chi=64, norm_method=0)),
    ("norm2", 6, 0.9, dict(Dmax=16, chi=64, norm_method=2)),
    ("norm0_l8", 8, 1.2, dict(Dmax=8, chi=32, norm_method=0)),
    ("norm2_l8", 8, 1.2, dict(Dmax=8, chi=32, norm_method=2)),
    ("nosvdopt", 8, 1.0, dict(Dmax=8, chi=32, svdopt=False)),
    ("noswapopt", 8, 1.0, dict(Dmax=8, chi=32, swapopt=False)),
    ("cutbond", 6, 0.9, dict(Dmax=16, chi=64, cut_bond=True)),
    ("compress", 8, 1.0, dict(Dmax=4, chi=16, compress=True)),
    ("compress_nosvdopt", 8, 1.0, dict(Dmax=4, chi=16, compress=True, svdopt=False)),
    ("select0_noreverse_norm2", 8, 1.0, dict(Dmax=8, chi=32, select=0, reverse=False, norm_method=2)),
    ("select2_compress_norm0", 8, 1.0, dict(Dmax=8, chi=32, select=2, compress=True, norm_method=0)),
]


@pytest.mark.parametrize("name,L,beta,kw", CASES, ids=[c[0] for c in CASES])
def test_option_trace_parity(catn, name, L, beta, kw):
    r = np.random.default_rng(zlib.crc32(name.encode()) % 1000)
    e = X.square_edges(L)
    w, h = r.normal(size=len(e)), r.normal(0, 0.1, L * L)
    ON.TRACE = []
    ref = OI.ising_network(L * L, e, w, h, beta, **kw)
    lz, err, psi = ON.contraction(ref)
    orows = oracle_rows(ON.TRACE)
    ON.TRACE = None
    tn = catn.ising_network(L * L, e, w, h, beta, **kw)
    lnZ, derr, dpsi = catn.contraction(tn, trace=True)
    rows = [tuple(int(x) for x in row[:7]) for row in tn.trace]
    assert rows == orows
    assert abs(lnZ - lz) / (L * L) <= 1e-10
    assert dpsi == psi
    assert tn.maxdim_intermediate == ref.maxdim_intermediate
    assert abs(derr - err) <= 1e-12 + 1e-6 * abs(err)


@pytest.mark.parametrize("sel", [0, 1, 2])
@pytest.mark.parametrize("rev", [False, True])
@pytest.mark.parametrize("comp", [False, True])
def test_exact_mode_options_trace_parity(catn, sel, rev, comp):
    """Exact mode (Dmax < 0) over select x reverse x compress on a 4x4 lattice:
    trace identical and lnZ equal to the row transfer matrix at rtol 1e-9."""
    r = np.random.default_rng(31 + 6 * sel + 2 * rev + comp)
    L = 4
    e = X.square_edges(L)
    w, h = r.normal(size=len(e)), r.normal(0, 0.1, L * L)
    kw = dict(Dmax=-1, chi=100000, select=sel, reverse=rev, compress=comp)
    ON.TRACE = []
    ref = OI.ising_network(L * L, e, w, h, 0.8, **kw)
    lz, _, _ = ON.contraction(ref)
    orows = oracle_rows(ON.TRACE)
    ON.TRACE = None
    tn = catn.ising_network(L * L, e, w, h, 0.8, **kw)
    lnZ, _, _ = catn.contraction(tn, trace=True)
    assert [tuple(int(x) for x in row[:7]) for row in tn.trace] == orows
    assert abs(lnZ - lz) / (L * L) <= 1e-10
    assert lnZ == pytest.approx(X.square_transfer_lnZ(L, L, e, w, h, 0.8), rel=1e-9)
