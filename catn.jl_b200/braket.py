"""``braket_network`` mirror over libcatn_b200 (reference ``src/braket.jl``).

``braket_network(tensors, ixs; chi, cutoff, norm_method, svdopt, swapopt,
seed)`` builds the double-layer network <psi|psi> of a real ket state; the
label analysis runs in the C library on the host, the BraKet nodes are built
and contracted on the device.  ``contraction(bk)`` returns
``(lnZ, error, psi)`` with ``<psi|psi> = exp(lnZ) * psi``.

``loops=True`` (no reference counterpart; the reference rejects a cyclic
virtual-bond graph) contracts loopy states such as PEPS: each pair of doubled
bonds that an eat makes parallel is fused, ket with ket and bra with bra.
"""
import ctypes as ct

import numpy as np

from . import _lib as L
from .network import TensorNetwork


class BraKetNetwork(TensorNetwork):
    """``BraKetNetwork`` (braket.jl:335-349) of ``braket_network(tensors, ixs)``."""

    def __init__(self, tensors, ixs, chi=64, cutoff=1e-15, norm_method=1, svdopt=True, swapopt=True, seed=1,
                 loops=False):
        self.kind = "braket"
        if len(tensors) != len(ixs):
            raise ValueError("braket_network: length(tensors) != length(ixs)")
        ts = []
        for t in tensors:
            a = np.asarray(t)
            if np.iscomplexobj(a):
                raise NotImplementedError("complex tensors are not supported by the device engine yet")
            ts.append(np.asarray(a, dtype=np.float64))
        ids = {}
        labels = []
        for k, ix in enumerate(ixs):
            if len(ix) != ts[k].ndim:
                raise ValueError(f"braket_network: tensor {k + 1} has {ts[k].ndim} axes but {len(ix)} labels")
            for lbl in ix:
                ids.setdefault(lbl, len(ids) + 1)
                labels.append(ids[lbl])
        self.tensors = ts
        self.labels = np.array(labels or [0], dtype=np.int32)
        self.n = len(ts)
        self.beta = 1.0
        # the C ABI takes the keyword set of TensorNetwork; Dmax is unused here
        self.params = dict(Dmax=-1, chi=chi, cutoff=cutoff, norm_method=norm_method, select=2, reverse=False,
                           svdopt=svdopt, swapopt=swapopt, compress=False, cut_bond=False, seed=seed,
                           braket_loops=bool(loops))
        self.neighbors = [list(ix) for ix in ixs]   # trace sizing only
        self.num_isolated = 0
        self._reset_outputs()
        self._dev = None
        _validate(ixs, loops)   # the reference's constructor errors (braket.jl:377-421), before any device work

    def _create(self, lib, p, arena):
        ndims = np.array([t.ndim for t in self.tensors], dtype=np.int32)
        dims = np.array([d for t in self.tensors for d in t.shape] or [0], dtype=np.int64)
        data = np.ascontiguousarray(np.concatenate([np.ravel(t, order="F") for t in self.tensors]))
        h = ct.c_void_p()
        L.check(lib, lib.catn_braket_create(ct.byref(p), self.n, L.ptr(ndims), L.ptr(dims), L.ptr(data),
                                            L.ptr(self.labels), int(arena), ct.byref(h)))
        return h


def _validate(ixs, loops=False):
    count, owners = {}, {}
    for k, ix in enumerate(ixs):
        for lbl in ix:
            count[lbl] = count.get(lbl, 0) + 1
            owners.setdefault(lbl, []).append(k)
    for lbl, c in count.items():
        if c > 2:
            raise ValueError(f"braket_network: label {lbl} appears {c} times (expected 1 or 2)")
    for k, ix in enumerate(ixs):
        nphys = sum(1 for lbl in ix if count[lbl] == 1)
        if nphys != 1:
            raise ValueError(f"braket_network: tensor {k + 1} has {nphys} physical (open) labels, expected 1")
    parent = list(range(len(ixs)))

    def root(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    pairs = set()
    for lbl, o in owners.items():
        if len(o) == 2 and loops:
            key = (min(o), max(o))
            if key in pairs:
                raise ValueError(f"braket_network: tensors {key[0] + 1} and {key[1] + 1} share more than one label "
                                 "(parallel bonds are not supported)")
            pairs.add(key)
        elif len(o) == 2:
            a, b = root(o[0]), root(o[1])
            if a == b:
                raise ValueError("braket_network: virtual-bond graph contains a cycle — cyclic graphs are not "
                                 "supported in v1")
            parent[a] = b


def braket_network(tensors, ixs, chi=64, cutoff=1e-15, norm_method=1, svdopt=True, swapopt=True, seed=1,
                   loops=False):
    """``braket_network`` (braket.jl:369-508); ``loops=True`` accepts cyclic
    virtual-bond graphs (fusing parallel doubled bonds as they form)."""
    return BraKetNetwork(tensors, ixs, chi=chi, cutoff=cutoff, norm_method=norm_method, svdopt=svdopt,
                         swapopt=swapopt, seed=seed, loops=loops)
