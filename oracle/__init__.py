"""CPU oracle for the CATN ``contraction!`` hot path.

TEST INFRASTRUCTURE ONLY.  This package is a line-by-line numpy restatement of
the reference Julia package xuanzhaogao/CATN.jl v0.1.0 (``src/linalg_utils.jl``,
``src/mps_node.jl``, ``src/tensor_network.jl``, ``src/ising.jl``).  It is the
checker that the CUDA library is compared against, and the timed CPU baseline
in ``bench.py``.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline legs of ``bench.py`` may import it; the product library
(``catn_b200``) never does.

Conventions kept from the reference:
  * every MPS site is a rank-3 array ``(left, phys, right)`` and every reshape
    is column-major (``order='F'``), so index arithmetic matches Julia's;
  * neighbour positions are 1-based (0 = "not found"), node ids are 1-based,
    open legs are negative sentinels;
  * LAPACK drivers are the reference's: ``gesdd`` with a ``gesvd`` fallback
    (``numpy.linalg.svd`` / ``scipy.linalg.svd``) and Householder ``geqrf``.

Parity pins: the reference ships no golden vectors (its tests draw random
inputs).  The oracle is pinned instead against the reference's known-answer
tests -- Ising chain vs transfer matrix, triangle vs brute force,
magnetization/correlation vs brute force, isolated spins, exact mode vs dense
einsum -- restated in ``tests/test_oracle_*.py``, and against independent exact
checkers (``oracle.exact``).  Julia is not available in this environment, so
the reference itself cannot be executed to produce fixtures.
"""
