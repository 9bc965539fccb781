"""Ising / spin-glass API mirror over libcatn_b200 (reference ``src/ising.jl``).

``ising_network`` builds the same MPS-form network as the reference
(ising.jl:20-227; the builder runs in the C library on the host, as the
reference's runs in Julia), and ``contraction`` contracts it on the device.
``magnetization`` / ``correlation`` keep the reference's pinning
definition (ising.jl:263-339) but contract all 1+2n or 1+4|E| pinned
networks in ONE persistent kernel launch instead of a host loop.
``IsingBatch`` is the batched entry point (many instances, one launch).

``gradient`` (and ``method="adjoint"`` of the two observables) replaces the
pinning loops with the device adjoint: one taped forward contraction and one
backward pass give d lnZ / d w_e = beta <s_i s_j> and d lnZ / d h_k =
beta <s_k> for every edge and spin at once (no reference counterpart; the
reference only has pinning).  ``IsingLnZ`` wraps it as a
``torch.autograd.Function``.
"""
import ctypes as ct

import numpy as np

from . import _lib as L
from .network import TensorNetwork, contraction, _Device


class IsingNetwork(TensorNetwork):
    """Partition-function network of ``ising_network(n, edges, weights,
    fields, beta; pos1, val1, pos2, val2, Dmax, chi, ...)``."""

    def __init__(self, n, edges, weights, fields, beta, pos1=0, val1=0, pos2=0, val2=0, Dmax=32, chi=32,
                 cutoff=1e-15, norm_method=1, select=1, reverse=True, svdopt=True, swapopt=True,
                 compress=False, cut_bond=False, seed=1, rsvd=0, rsvd_min_dim=0,
                 precision="fp64", svd_route="auto", ckpt_interval=0):
        self.kind = "ising"
        self.n = int(n)
        self.edges = np.asarray(edges, dtype=np.int32).reshape(-1, 2) if len(edges) else np.zeros((0, 2), np.int32)
        self.weights = np.asarray(weights, dtype=np.float64).reshape(-1)
        self.fields = np.asarray(fields, dtype=np.float64).reshape(-1)
        if self.fields.size != self.n:
            raise ValueError("fields must have one entry per spin")
        if self.weights.size != self.edges.shape[0]:
            raise ValueError("weights must have one entry per edge")
        self.beta = float(beta)
        self.pins = (int(pos1), int(val1), int(pos2), int(val2))
        self.params = dict(Dmax=Dmax, chi=chi, cutoff=cutoff, norm_method=norm_method, select=select,
                           reverse=reverse, svdopt=svdopt, swapopt=swapopt, compress=compress,
                           cut_bond=cut_bond, seed=seed, rsvd=rsvd,
                           rsvd_min_dim=rsvd_min_dim, precision=precision, svd_route=svd_route,
                           ckpt_interval=ckpt_interval)
        self.neighbors = [[0, 0] for _ in range(self.edges.shape[0])]   # trace sizing only
        deg = np.zeros(self.n + 1, int)
        for i, j in self.edges:
            deg[i] += 1
            deg[j] += 1
        self.num_isolated = int(np.sum(deg[1:] == 0))
        self._reset_outputs()
        self._dev = None

    def _create(self, lib, p, arena):
        h = ct.c_void_p()
        e = np.ascontiguousarray(self.edges.reshape(-1), dtype=np.int32)
        L.check(lib, lib.catn_ising_create(ct.byref(p), self.n, self.edges.shape[0], L.ptr(e),
                                           L.ptr(self.weights), L.ptr(self.fields), self.beta, *self.pins,
                                           int(arena), ct.byref(h)))
        return h


def ising_network(n, edges, weights, fields, beta, **kw):
    """``ising_network`` (ising.jl:20-227)."""
    return IsingNetwork(n, edges, weights, fields, beta, **kw)


def gradient(tn, ckpt_interval=None):
    """``(lnZ, dlnZ_dw, dlnZ_dh)`` of an Ising network from one forward
    contraction with a tape plus one backward pass, both on the device.
    ``dlnZ_dw[e] = beta <s_i s_j>``, ``dlnZ_dh[k] = beta <s_k>`` (exact up to
    the contraction's own truncations).  ``ckpt_interval`` (default: the
    network's) > 0 keeps a checkpoint every that many steps and recomputes
    the segments in the backward pass; the gradients are the same bit for
    bit.  Does not consume ``tn``."""
    if not isinstance(tn, IsingNetwork):
        raise TypeError("gradient: networks built by ising_network only")
    dev = tn._ensure_device()
    lib = L.load()
    res = L.Result()
    dw = np.zeros(max(tn.edges.shape[0], 1))
    dh = np.zeros(tn.n)
    k = tn.params.get("ckpt_interval", 0) if ckpt_interval is None else ckpt_interval
    L.check(lib, lib.catn_ising_grad(dev.handle, ct.byref(res), L.ptr(dw), L.ptr(dh), int(k)))
    return res.lnZ, dw[:tn.edges.shape[0]], dh


def free_energy(tn):
    """``free_energy(tn) -> (lnZ/n, -lnZ/(n beta))`` (ising.jl:239-244)."""
    lnZ, _, _ = contraction(tn)
    lps = lnZ / tn.n
    return lps, -lps / tn.beta


class IsingBatch:
    """Many Ising instances contracted in one persistent kernel launch.

    ``instances`` is a list of dicts with keys n, edges, weights, fields,
    beta and optional pos1/val1/pos2/val2; ``params`` are the keyword
    arguments shared by all instances.
    """

    def __init__(self, instances, slot_arena_bytes=0, max_slots=0, trace=False, **params):
        self.lib = L.load()
        nb = len(instances)
        n_nodes = np.array([int(d["n"]) for d in instances], dtype=np.int32)
        node_off = np.zeros(nb + 1, dtype=np.int64)
        edge_off = np.zeros(nb + 1, dtype=np.int64)
        edges, weights, fields, betas, pins = [], [], [], [], []
        for q, d in enumerate(instances):
            e = np.asarray(d["edges"], dtype=np.int32).reshape(-1, 2)
            edges.append(e.reshape(-1))
            weights.append(np.asarray(d["weights"], dtype=np.float64).reshape(-1))
            fields.append(np.asarray(d["fields"], dtype=np.float64).reshape(-1))
            betas.append(float(d["beta"]))
            pins.append([int(d.get("pos1", 0)), int(d.get("val1", 0)), int(d.get("pos2", 0)), int(d.get("val2", 0))])
            node_off[q + 1] = node_off[q] + n_nodes[q]
            edge_off[q + 1] = edge_off[q] + e.shape[0]
        self.n_nodes = n_nodes
        self._arrays = [n_nodes, node_off, edge_off,
                        np.ascontiguousarray(np.concatenate(edges) if edges else np.zeros(2), dtype=np.int32),
                        np.ascontiguousarray(np.concatenate(weights) if weights else np.zeros(1)),
                        np.ascontiguousarray(np.concatenate(fields)),
                        np.ascontiguousarray(np.array(betas)),
                        np.ascontiguousarray(np.array(pins, dtype=np.int32).reshape(-1))]
        p = L.make_params(trace=trace, **params)
        h = ct.c_void_p()
        a = self._arrays
        L.check(self.lib, self.lib.catn_ising_batch_create(ct.byref(p), nb, L.ptr(a[0]), L.ptr(a[1]), L.ptr(a[2]),
                                                           L.ptr(a[3]), L.ptr(a[4]), L.ptr(a[5]), L.ptr(a[6]),
                                                           L.ptr(a[7]), int(slot_arena_bytes), int(max_slots),
                                                           ct.byref(h)))
        self.handle = h
        self.size = nb
        self.results = (L.Result * nb)()

    @property
    def slots(self):
        return self.lib.catn_batch_slots(self.handle)

    @property
    def input_bytes(self):
        return self.lib.catn_batch_input_bytes(self.handle)

    def upload(self, stream=None):
        L.check(self.lib, self.lib.catn_batch_upload(self.handle, stream))

    def launch(self, stream=None):
        L.check(self.lib, self.lib.catn_batch_launch(self.handle, stream))

    def fetch(self, stream=None):
        L.check(self.lib, self.lib.catn_batch_results(self.handle, self.results, stream))
        return self.results

    def run(self):
        """Upload inputs, contract every instance, return per-instance results."""
        L.check(self.lib, self.lib.catn_batch_run(self.handle, self.results))
        return self.results

    def set_params(self, weights, fields, betas=None, stream=None):
        """New couplings, fields (and betas) for every instance, same lattices
        and pins: concatenated in instance order like the constructor's
        input.  Only these arrays go to the device, where the site tensors are
        rebuilt; ``launch`` then contracts the new networks (``upload``
        restores the networks given at construction)."""
        a = self._arrays
        w = np.ascontiguousarray(weights, dtype=np.float64).reshape(-1)
        h = np.ascontiguousarray(fields, dtype=np.float64).reshape(-1)
        if w.size != int(a[2][-1]) or h.size != int(a[1][-1]):
            raise ValueError(f"set_params: expected {int(a[2][-1])} weights and {int(a[1][-1])} fields, "
                             f"got {w.size} and {h.size}")
        b = None
        if betas is not None:
            b = np.ascontiguousarray(betas, dtype=np.float64).reshape(-1)
            if b.size != self.size:
                raise ValueError(f"set_params: expected {self.size} betas, got {b.size}")
        self._params_keep = (w, h, b)   # alive until the asynchronous copy has run
        L.check(self.lib, self.lib.catn_ising_batch_set_params(self.handle, L.ptr(w) if w.size else None, L.ptr(h),
                                                               L.ptr(b) if b is not None else None, stream))

    def randomize(self, seed, sigma_w=1.0, sigma_h=0.0, stream=None):
        """Disorder generated on the device: weights ~ sigma_w N(0,1), fields ~
        sigma_h N(0,1) (counter-based generator keyed by ``seed``), site
        tensors rebuilt there."""
        L.check(self.lib, self.lib.catn_ising_batch_randomize(self.handle, int(seed) & (2 ** 64 - 1),
                                                              float(sigma_w), float(sigma_h), stream))

    def params(self):
        """The device's current (weights, fields, betas), concatenated."""
        a = self._arrays
        w = np.zeros(max(int(a[2][-1]), 1))
        h = np.zeros(int(a[1][-1]))
        b = np.zeros(self.size)
        L.check(self.lib, self.lib.catn_ising_batch_get_params(self.handle, L.ptr(w), L.ptr(h), L.ptr(b)))
        return w[:int(a[2][-1])], h, b

    @property
    def param_bytes(self):
        return self.lib.catn_ising_batch_param_bytes(self.handle)

    def grad_launch(self, stream=None):
        """Upload and start the gradient run of every instance (one launch)."""
        L.check(self.lib, self.lib.catn_batch_grad_launch(self.handle, stream))

    def grad_fetch(self, stream=None):
        """Results and gradients of the last gradient run: (results, dlnZ_dw,
        dlnZ_dh), the gradients concatenated per instance."""
        a = self._arrays
        dw = np.zeros(max(int(a[2][-1]), 1))
        dh = np.zeros(int(a[1][-1]))
        L.check(self.lib, self.lib.catn_batch_grad_results(self.handle, self.results, L.ptr(dw), L.ptr(dh), stream))
        return self.results, dw[:int(a[2][-1])], dh

    def grad(self):
        """Gradient run of every instance; per instance (lnZ, dlnZ_dw, dlnZ_dh)."""
        self.grad_launch()
        res, dw, dh = self.grad_fetch()
        a = self._arrays
        return [(res[q].lnZ, dw[a[2][q]:a[2][q + 1]], dh[a[1][q]:a[1][q + 1]]) for q in range(self.size)]

    def lnZ(self):
        return np.array([r.lnZ for r in self.results])

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                self.lib.catn_batch_destroy(self.handle)
        except Exception:
            pass
        self.handle = None


def _pinned_batch(n, edges, weights, fields, beta, pins, **kw):
    insts = [dict(n=n, edges=edges, weights=weights, fields=fields, beta=beta,
                  pos1=p[0], val1=p[1], pos2=p[2], val2=p[3]) for p in pins]
    b = IsingBatch(insts, **kw)
    b.run()
    return b.lnZ()


def magnetization(n, edges, weights, fields, beta, method="pinning", **kw):
    """<s_k> by spin pinning (ising.jl:263-290): 1 + 2n contractions, all in
    one launch; ``method="adjoint"`` gives d lnZ / d h / beta from one
    gradient run instead."""
    if method == "adjoint":
        _, _, dh = gradient(ising_network(n, edges, weights, fields, beta, **kw))
        return dh / beta
    if method != "pinning":
        raise ValueError("method must be 'pinning' or 'adjoint'")
    pins = [(0, 0, 0, 0)] + [(k, v, 0, 0) for k in range(1, n + 1) for v in (1, 2)]
    lz = _pinned_batch(n, edges, weights, fields, beta, pins, **kw)
    p = np.exp(lz[1:] - lz[0]).reshape(n, 2)
    return p[:, 1] - p[:, 0]


def correlation(n, edges, weights, fields, beta, method="pinning", **kw):
    """<s_i s_j> per edge by pinning both ends (ising.jl:309-339): 1 + 4|E|
    contractions, one launch; ``method="adjoint"`` gives d lnZ / d w / beta
    from one gradient run instead."""
    if method == "adjoint":
        _, dw, _ = gradient(ising_network(n, edges, weights, fields, beta, **kw))
        return dw / beta
    if method != "pinning":
        raise ValueError("method must be 'pinning' or 'adjoint'")
    pins = [(0, 0, 0, 0)]
    for (m, nn) in edges:
        for v1 in (1, 2):
            for v2 in (1, 2):
                pins.append((int(m), v1, int(nn), v2))
    lz = _pinned_batch(n, edges, weights, fields, beta, pins, **kw)
    p = np.exp(lz[1:] - lz[0]).reshape(len(edges), 2, 2)
    return p[:, 0, 0] - p[:, 0, 1] - p[:, 1, 0] + p[:, 1, 1]


def _make_autograd():
    import torch

    class IsingLnZ(torch.autograd.Function):
        """lnZ(weights, fields) of ``ising_network(n, edges, weights, fields,
        beta, **params)`` as a differentiable function: forward and backward
        both come from one device gradient run (the Python counterpart of the
        ChainRulesCore ``rrule`` a Julia caller would attach)."""

        @staticmethod
        def forward(ctx, weights, fields, n, edges, beta, params):
            lnZ, dw, dh = gradient(ising_network(n, edges, weights.detach().cpu().double().numpy(),
                                                 fields.detach().cpu().double().numpy(), beta, **params))
            ctx.save_for_backward(torch.from_numpy(dw).to(weights), torch.from_numpy(dh).to(fields))
            return weights.new_tensor(lnZ)

        @staticmethod
        def backward(ctx, g):
            dw, dh = ctx.saved_tensors
            return g * dw, g * dh, None, None, None, None

    return IsingLnZ


def ising_lnZ(weights, fields, n, edges, beta, **params):
    """Differentiable lnZ (torch tensors in, torch scalar out); see
    ``IsingLnZ``."""
    global IsingLnZ
    if IsingLnZ is None:
        IsingLnZ = _make_autograd()
    return IsingLnZ.apply(weights, fields, n, edges, beta, params)


IsingLnZ = None
