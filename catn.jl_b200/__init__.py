"""catn_b200: B200-native implementation of the CATN.jl ``contraction!`` hot path.

Public API (mirrors CATN.jl's exports for this path, src/CATN.jl:15-32):

    TensorNetwork, contraction (= contraction!), result_tensor, adapt, B200,
    ising_network, free_energy, magnetization, correlation, IsingBatch,
    gradient, ising_lnZ (device adjoint; no reference counterpart),
    tc_matmul (the split-precision tensor-core product; no reference counterpart),
    braket_network, BraKetNetwork

All compute runs in ``libcatn_b200.so`` (sm_100a).  Import this directory as
the package ``catn_b200`` (``__graft_entry__.load_package()`` does it).
"""
from ._lib import CatnError, load as load_library
from .braket import BraKetNetwork, braket_network
from .network import (B200, TensorNetwork, adapt, contraction, cut_bondim, cut_bondim_opt, release_cached_memory,
                      result_tensor, tc_matmul)
from .ising import (IsingBatch, IsingNetwork, correlation, free_energy, gradient, ising_lnZ, ising_network,
                    magnetization)

__all__ = ["B200", "BraKetNetwork", "CatnError", "IsingBatch", "IsingNetwork", "TensorNetwork", "adapt", "braket_network", "contraction",
           "correlation", "free_energy", "gradient", "ising_lnZ", "ising_network", "load_library",
           "magnetization", "result_tensor", "tc_matmul", "cut_bondim", "cut_bondim_opt", "release_cached_memory"]
