"""Ising / spin-glass network builder and pinning observables (oracle; test infrastructure).

Restates ``src/ising.jl`` of CATN.jl.
"""
import math

import numpy as np

from . import mps as M
from .network import TensorNetwork, contraction


def ising_network(n, edges, weights, fields, beta, pos1=0, val1=0, pos2=0, val2=0, Dmax=32,
                  chi=32, cutoff=1e-15, norm_method=1, select=1, reverse=True, svdopt=True,
                  swapopt=True, compress=False, cut_bond=False, seed=1):
    """Build the partition-function network directly in MPS form (ising.jl:20-227).

    Edge ``(i, j)`` (1-based) puts ``B = exp(beta w s_i s_j)`` on node ``i`` and
    the identity on node ``j``; each node becomes a chain of one site per
    incident edge (leaf / first / last / interior layouts), with the field
    folded into the first (or leaf) site.  ``pos*/val*`` pin a spin by zeroing
    one spin component (val 1 zeroes +1, val 2 zeroes -1).
    """
    degree = [0] * (n + 1)
    for (i, j) in edges:
        degree[i] += 1
        degree[j] += 1
    nodes = {k: M.MPSNode([], [], 0, chi, cutoff, norm_method, svdopt, swapopt)
             for k in range(1, n + 1)}
    spin = np.array([1.0, -1.0])
    R = np.eye(2)

    def site(node, deg, field, Q):
        if deg == 1:
            mat = np.diag(field) @ Q
            return M.rs(mat.sum(axis=0), 1, 2, 1)
        if not node.neighbor:
            return M.rs((np.diag(field) @ Q).T, 1, 2, 2)
        if len(node.neighbor) == deg - 1:
            return M.rs(Q.copy(), 2, 2, 1)
        t3 = np.zeros((2, 2, 2))
        t3[:, 0, :] = np.diag(Q[:, 0])
        t3[:, 1, :] = np.diag(Q[:, 1])
        return t3

    for e, (i, j) in enumerate(edges):
        si, sj = spin.copy(), spin.copy()
        if i == pos1:
            si[val1 - 1] = 0.0
        elif i == pos2:
            si[val2 - 1] = 0.0
        if j == pos1:
            sj[val1 - 1] = 0.0
        elif j == pos2:
            sj[val2 - 1] = 0.0
        Mij = np.outer(si, sj)
        w = float(weights[e])
        B = np.exp(beta * w * Mij)
        fi = np.exp(beta * float(fields[i - 1]) * si)
        nodes[i].mps.append(site(nodes[i], degree[i], fi, B))
        nodes[i].neighbor.append(j)
        fj = np.exp(beta * float(fields[j - 1]) * sj)
        nodes[j].mps.append(site(nodes[j], degree[j], fj, R))
        nodes[j].neighbor.append(i)
    for k in range(1, n + 1):
        if degree[k] == 0:
            hk = float(fields[k - 1])
            val = math.exp(beta * hk) + math.exp(-beta * hk)
            nodes[k].mps.append(np.full((1, 1, 1), val))
    for node in nodes.values():
        node.cano = len(node.mps)
    num_isolated = sum(1 for k in range(1, n + 1) if not nodes[k].neighbor)
    return TensorNetwork(nodes, Dmax=Dmax, chi=chi, cutoff=cutoff, norm_method=norm_method,
                         select=select, reverse=reverse, svdopt=svdopt, swapopt=swapopt,
                         compress=compress, cut_bond=cut_bond, seed=seed, n=n, beta=beta,
                         num_isolated=num_isolated)


def free_energy(tn):
    """``(lnZ/n, -lnZ/(n beta))`` (ising.jl:239-244)."""
    lnZ, _, _ = contraction(tn)
    lps = lnZ / tn.n
    return lps, -lps / tn.beta


def magnetization(n, edges, weights, fields, beta, **kw):
    """<s_k> by pinning each spin to each value: 1 + 2n contractions (ising.jl:263-290)."""
    lnZ_total, _, _ = contraction(ising_network(n, edges, weights, fields, beta, **kw))
    mag = np.zeros(n)
    for k in range(1, n + 1):
        lz = np.zeros(2)
        for val in (1, 2):
            lz[val - 1], _, _ = contraction(
                ising_network(n, edges, weights, fields, beta, pos1=k, val1=val, **kw))
        p = np.exp(lz - lnZ_total)
        mag[k - 1] = p[1] - p[0]
    return mag


def correlation(n, edges, weights, fields, beta, **kw):
    """<s_i s_j> per edge by pinning both ends: 1 + 4|E| contractions (ising.jl:309-339)."""
    lnZ_total, _, _ = contraction(ising_network(n, edges, weights, fields, beta, **kw))
    cor = np.zeros(len(edges))
    for e, (m, nn) in enumerate(edges):
        lz = np.zeros((2, 2))
        for v1 in (1, 2):
            for v2 in (1, 2):
                lz[v1 - 1, v2 - 1], _, _ = contraction(
                    ising_network(n, edges, weights, fields, beta, pos1=m, val1=v1, pos2=nn,
                                  val2=v2, **kw))
        p = np.exp(lz - lnZ_total)
        cor[e] = p[0, 0] - p[0, 1] - p[1, 0] + p[1, 1]
    return cor
