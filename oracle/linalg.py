"""Truncated / randomized SVD and thin-Q helpers (oracle; test infrastructure).

Restates ``src/linalg_utils.jl`` of CATN.jl.
"""
import numpy as np
import scipy.linalg

# Optional per-call log of every SVD the oracle performs: (tag, m, n, kept).
SVD_LOG = None


def _svd_full(A):
    """``svd(A)`` with the QRIteration fallback (linalg_utils.jl:16-21).

    numpy's ``linalg.svd`` is LAPACK gesdd (divide and conquer), the driver
    Julia's ``svd`` uses; on failure fall back to gesvd (QR iteration).
    Returns (U, S, V) with ``A = U diag(S) V^H``.
    """
    try:
        U, S, Vh = np.linalg.svd(A, full_matrices=False)
    except np.linalg.LinAlgError:
        U, S, Vh = scipy.linalg.svd(A, full_matrices=False, lapack_driver="gesvd")
    return U, S, Vh.conj().T


def tsvd(A, cutoff=1e-15, maxdim=None, tag="tsvd"):
    """Truncated thin SVD, ``A ~ U diag(S) V^H`` (linalg_utils.jl:15-28).

    ``nkeep = count(S > cutoff)``; zero kept becomes one; capped at ``maxdim``.
    The fourth return value is the sum of the discarded singular values
    (not their squares), as in the reference.
    """
    U, S, V = _svd_full(A)
    nfull = S.shape[0]
    nkeep = int(np.count_nonzero(S > cutoff))
    if nkeep == 0:
        nkeep = 1
    else:
        nkeep = min(nkeep, nfull if maxdim is None else maxdim, nfull)
    discarded = float(np.sum(S[nkeep:nfull])) if nkeep < nfull else 0.0
    if SVD_LOG is not None:
        SVD_LOG.append((tag, A.shape[0], A.shape[1], nkeep))
    return U[:, :nkeep], S[:nkeep], V[:, :nkeep], discarded


def thin_qr(A):
    """Householder QR with the thin Q materialised (linalg_utils.jl:32-37)."""
    Q, R = np.linalg.qr(A, mode="reduced")
    return Q, R


def rsvd(A, k, oversample=10, power=10, rng=None):
    """Randomized SVD (linalg_utils.jl:44-58).

    ``p = min(n, oversample*k)`` -- the oversampling is multiplicative in the
    reference; ``power`` rounds of ``Y <- thinQ(A (A^H Y))``.  The reference
    draws the sketch from Julia's global RNG (unseeded from ``contraction!``),
    so this restatement can only match it in distribution, not bit for bit.
    """
    if rng is None:
        rng = np.random.default_rng(0)
    n = A.shape[1]
    p = min(n, oversample * k)
    G = rng.standard_normal((n, p))
    if np.iscomplexobj(A):
        G = G + 1j * rng.standard_normal((n, p))
    Y = A @ G
    for _ in range(power):
        M = A @ (A.conj().T @ Y)
        Y, _r = np.linalg.qr(M, mode="reduced")
    Q, _r = np.linalg.qr(Y, mode="reduced")
    B = Q.conj().T @ A
    Ub, S, V = _svd_full(B)
    kk = min(k, Ub.shape[1])
    return (Q @ Ub)[:, :kk], S[:kk], V[:, :kk]
