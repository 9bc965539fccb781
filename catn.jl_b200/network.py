"""Host mirror of the reference's network API over libcatn_b200.

Reference: ``src/tensor_network.jl`` (TensorNetwork, contraction!,
result_tensor) and ``src/adapt.jl`` (the device-move hook).  The Python
names drop Julia's ``!``: ``contraction`` is ``contraction!``.

A ``TensorNetwork`` is a host description (labels resolved into neighbour
lists exactly as tensor_network.jl:56-116 does); ``adapt(B200, tn)`` moves it
to HBM (one device-resident ``catn_net``) and ``contraction(tn)`` runs the
whole contraction on the GPU in one kernel launch.
"""
import ctypes as ct

import numpy as np

from . import _lib as L

B200 = "b200"   # adapt target, the counterpart of `CuArray` in adapt(CuArray, tn)


class _Device:
    """Owns one catn_net handle."""

    def __init__(self, handle):
        self.handle = handle

    def __del__(self):
        try:
            if self.handle:
                L.load().catn_net_destroy(self.handle)
        except Exception:
            pass
        self.handle = None


class TensorNetwork:
    """``TensorNetwork(tensors, ixs; Dmax, chi, cutoff, norm_method, select,
    reverse, svdopt, swapopt, compress, cut_bond, seed)``
    (tensor_network.jl:41-140).

    - a label shared by exactly two tensors becomes a bond;
    - a label appearing once becomes an open leg (negative sentinel);
    - a label appearing more than twice, or twice in one tensor, raises.
    """

    def __init__(self, tensors, ixs, Dmax=32, chi=32, cutoff=1e-15, norm_method=1, select=1,
                 reverse=True, svdopt=True, swapopt=True, compress=False, cut_bond=False, seed=1, rsvd=0, rsvd_min_dim=0,
                 precision="fp64", svd_route="auto"):
        n = len(tensors)
        if len(ixs) != n:
            raise ValueError("tensors and ixs must have the same length")
        for t, ix in enumerate(ixs):
            seen = set()
            for lbl in ix:
                if lbl in seen:
                    raise ValueError(f"Self-loop detected: label {lbl} appears twice in tensor {t + 1}'s index list")
                seen.add(lbl)
        label_map = {}
        for t, ix in enumerate(ixs):
            if np.ndim(tensors[t]) != len(ix):
                raise ValueError(f"tensor {t + 1} has {np.ndim(tensors[t])} legs but {len(ix)} labels")
            for k, lbl in enumerate(ix):
                label_map.setdefault(lbl, []).append((t, k))
        for lbl, occ in label_map.items():
            if len(occ) > 2:
                raise ValueError(f"Label {lbl} appears in {len(occ)} tensors (max 2 allowed)")
        nbr = [[0] * len(ix) for ix in ixs]
        sentinel = 0
        for lbl, occ in label_map.items():
            if len(occ) == 2:
                (t1, k1), (t2, k2) = occ
                nbr[t1][k1] = t2 + 1
                nbr[t2][k2] = t1 + 1
            else:
                sentinel -= 1
                t, k = occ[0]
                nbr[t][k] = sentinel
        self.kind = "dense"
        if any(np.iscomplexobj(t) for t in tensors):
            raise NotImplementedError("complex tensors are not supported by the device engine yet")
        self.tensors = [np.asarray(t, dtype=np.float64) for t in tensors]
        self.neighbors = nbr
        self.n = n
        self.beta = 1.0
        self.params = dict(Dmax=Dmax, chi=chi, cutoff=cutoff, norm_method=norm_method, select=select,
                           reverse=reverse, svdopt=svdopt, swapopt=swapopt, compress=compress,
                           cut_bond=cut_bond, seed=seed, rsvd=rsvd,
                           rsvd_min_dim=rsvd_min_dim, precision=precision, svd_route=svd_route)
        self.num_isolated = sum(1 for v in nbr if all(x < 0 for x in v))
        self._reset_outputs()
        self._dev = None

    def _reset_outputs(self):
        self.lnZ = 0.0
        self.sign = 1.0
        self.psi = 1.0
        self.error = 0.0
        self.maxdim_intermediate = -1
        self.trace = None
        self.result = None

    # -- device move (adapt.jl:12-24) -------------------------------------------
    def _create(self, lib, p, arena):
        ndims = np.array([t.ndim for t in self.tensors], dtype=np.int32)
        dims = np.array([d for t in self.tensors for d in t.shape] or [0], dtype=np.int64)
        data = np.concatenate([np.ravel(t, order="F") for t in self.tensors]) if self.tensors else np.zeros(1)
        data = np.ascontiguousarray(data, dtype=np.float64)
        nbrs = np.array([v for ix in self.neighbors for v in ix] or [0], dtype=np.int32)
        h = ct.c_void_p()
        L.check(lib, lib.catn_net_create_dense(ct.byref(p), self.n, L.ptr(ndims), L.ptr(dims), L.ptr(data),
                                               L.ptr(nbrs), int(arena), ct.byref(h)))
        return h

    def _ensure_device(self, trace=False, arena_bytes=0):
        if self._dev is None:
            lib = L.load()
            p = L.make_params(trace=trace, **self.params)
            self._dev = _Device(self._create(lib, p, arena_bytes))
            self._trace_on = trace
        return self._dev


def adapt(to, tn, trace=False, arena_bytes=0):
    """``adapt(CuArray, tn)`` counterpart (adapt.jl:6-24): copy the network
    into HBM.  Only the B200 target is supported; the element type is FP64."""
    if to not in (B200, "cuda", "b200"):
        raise ValueError(f"adapt: unsupported target {to!r}")
    tn._ensure_device(trace=trace, arena_bytes=arena_bytes)
    return tn


def contraction(tn, trace=False, arena_bytes=0):
    """``contraction!(tn) -> (lnZ, error, psi)`` (tensor_network.jl:556-717).

    Consumes the network (as the reference does); afterwards
    ``result_tensor(tn)`` gives the surviving open-leg tensor.
    ``trace=True`` also records the per-step integer trace in ``tn.trace``
    (an (nsteps, 8) int32 array; see include/catn_b200.h).
    """
    dev = tn._ensure_device(trace=trace, arena_bytes=arena_bytes)
    lib = L.load()
    res = L.Result()
    cap = 0
    tr = None
    if trace:
        cap = 4 * sum(len(ix) for ix in getattr(tn, "neighbors", [[0]])) + 64
        tr = np.zeros(8 * cap, dtype=np.int32)
    L.check(lib, lib.catn_contract(dev.handle, ct.byref(res), L.ptr(tr), cap))
    tn.lnZ, tn.error, tn.psi, tn.sign = res.lnZ, res.err, res.psi, res.sign
    tn.maxdim_intermediate = res.maxdim
    tn.result = res
    if trace:
        tn.trace = tr[: 8 * min(res.nsteps, cap)].reshape(-1, 8).copy()
    return res.lnZ, res.err, res.psi


def _cut(tn, i, idx_j_in_i, opt):
    if tn.result is not None:
        raise ValueError("network already contracted (contraction! consumes tn)")
    dev = tn._ensure_device()
    lib = L.load()
    err = ct.c_double()
    L.check(lib, lib.catn_cut_bondim(dev.handle, int(i), int(idx_j_in_i), 1 if opt else 0, ct.byref(err)))
    return err.value


def cut_bondim(tn, i, idx_j_in_i):
    """``cut_bondim!(tn, i, idx_j_in_i) -> error`` (tensor_network.jl:342-388):
    truncate the bond between node ``i`` and its neighbour on leg
    ``idx_j_in_i`` to ``Dmax`` singular values of the plain product of the
    two bond sites (no canonicalisation, no QR pre-reduction), on the
    device.  Returns the discarded singular-value sum; a later
    ``contraction(tn)`` contracts the cut network."""
    return _cut(tn, i, idx_j_in_i, False)


def cut_bondim_opt(tn, i, idx_j_in_i):
    """``cut_bondim_opt!(tn, i, idx_j_in_i) -> error``
    (tensor_network.jl:399-477): the same cut after canonicalising both
    nodes to the shared leg, with QR pre-reduction of both sides."""
    return _cut(tn, i, idx_j_in_i, True)


def result_tensor(tn):
    """``result_tensor(tn)`` (tensor_network.jl:517-523): dense tensor of the
    single surviving open-leg node (legs in its final MPS order); a 0-d one()
    for a closed network."""
    if tn._dev is None or tn.result is None:
        raise ValueError("result_tensor: contract the network first")
    lib = L.load()
    numel = ct.c_int64()
    nd = ct.c_int32()
    dims = np.zeros(64, dtype=np.int64)
    L.check(lib, lib.catn_result_tensor(tn._dev.handle, None, 0, ct.byref(numel), ct.byref(nd), L.ptr(dims)))
    if nd.value == 0:
        return np.ones(())
    out = np.zeros(int(numel.value), dtype=np.float64)
    L.check(lib, lib.catn_result_tensor(tn._dev.handle, L.ptr(out), out.size, ct.byref(numel), ct.byref(nd),
                                        L.ptr(dims)))
    return out.reshape(tuple(int(d) for d in dims[: nd.value]), order="F")


def tc_matmul(A, B):
    """``A @ B`` of two FP64 matrices on the tensor cores in the
    split-precision form (catn_tc_matmul: TF32 hi/lo parts, three tcgen05
    products per pair, FP32 accumulation; about 1e-6 of |A| |B|)."""
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    if A.ndim != 2 or B.ndim != 2 or A.shape[1] != B.shape[0]:
        raise ValueError("tc_matmul: shapes do not match")
    M, K = A.shape
    N = B.shape[1]
    C = np.zeros((M, N), dtype=np.float64, order="F")
    lib = L.load()
    L.check(lib, lib.catn_tc_matmul(M, N, K, L.ptr(A), L.ptr(B), L.ptr(C)))
    return C


def release_cached_memory():
    """Free the device and pinned host blocks the library keeps from
    destroyed networks and batches (``catn_release_cached_memory``), e.g.
    before handing the memory to another library.  Returns the device bytes
    that were kept."""
    lib = L.load()
    kept = int(lib.catn_cached_bytes(0))
    L.check(lib, lib.catn_release_cached_memory())
    return kept
