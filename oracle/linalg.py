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


def _splitmix64(x):
    """SplitMix64 mixing function (Steele, Lea and Flood, 2014) on uint64
    arrays (wrapping arithmetic)."""
    x = x + np.uint64(0x9E3779B97F4A7C15)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def counter_normal(seed, stream, index):
    """Standard normals from (seed, stream, index): SplitMix64 on a Weyl
    sequence of the counter and the Box-Muller transform of two 53-bit
    uniforms -- the generator the engine draws its rsvd sketch and device
    disorder from (csrc/ising_build.cuh, disorder_normal)."""
    index = np.asarray(index, dtype=np.uint64)
    key = _splitmix64(np.array([seed], dtype=np.uint64) ^ (np.array([stream], dtype=np.uint64)
                                                           * np.uint64(0xD1B54A32D192ED03)))[0]
    a = _splitmix64(key + np.uint64(2) * index)
    b = _splitmix64(key + np.uint64(2) * index + np.uint64(1))
    u1 = ((a >> np.uint64(11)) + np.uint64(1)).astype(np.float64) * (1.0 / 9007199254740992.0)
    u2 = (b >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(6.283185307179586 * u2)


def rsvd(A, k, oversample=10, power=10, rng=None, sketch=None):
    """Randomized SVD (linalg_utils.jl:44-58).

    ``p = min(n, oversample*k)`` -- the oversampling is multiplicative in the
    reference; ``power`` rounds of ``Y <- thinQ(A (A^H Y))``.  The reference
    draws the sketch from Julia's global RNG (unseeded from ``contraction!``),
    so this restatement can only match it in distribution, not bit for bit;
    ``sketch`` (n x p) supplies the Gaussian matrix instead.
    """
    if rng is None:
        rng = np.random.default_rng(0)
    n = A.shape[1]
    p = min(n, oversample * k)
    if sketch is not None:
        G = sketch
    else:
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
