"""vqemps: B200-native matrix-product-state engine for the Graph-VQE hot path.

Energies (shared-prefix transfer sweeps), SVD gate application (FP64 one-sided
Jacobi, zero cutoff, bond <= 16), the exact adjoint gradient and perfect
sampling run in hand-written sm_100a kernels behind the C ABI of
include/vqemps.h. Python only moves torch tensors and calls that ABI.
"""
from ._lib import EngineError
from .engine import Engine, Hamiltonian, PartitionSet, counts, unpack_bits

__all__ = ["Engine", "EngineError", "Hamiltonian", "PartitionSet", "counts", "unpack_bits"]
