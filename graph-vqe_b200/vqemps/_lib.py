"""ctypes binding of the engine's C ABI (include/vqemps.h).

The shared library is built in-tree (``graph-vqe_b200/vqemps/libvqemps.so``) by
``vqemps.build``; there is no fallback implementation: every entry point raises
if the library is missing.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

LIB_NAME = "libvqemps.so"
LIB_PATH = Path(__file__).resolve().parent / LIB_NAME

OK, INSUFFICIENT_BOND, NONFINITE_SVD, INVALID, CUDA_ERROR, TIMEOUT = range(6)

GATES = dict(rx=0, ry=1, rz=2, h=3, x=4, y=5, z=6, s=7, sdg=8, cx=9, u1=10, u2=11, swap=12)
INITIAL = {None: 0, "0": 0, "1": 1, "+": 2, "-": 3}
RNG = dict(splitmix=0, philox=1)
SHOT_MODES = dict(shared=0, plugin=1)

# Exported symbols of include/vqemps.h (checked by the CPU test suite).
SYMBOLS = (
    "vqemps_create", "vqemps_destroy", "vqemps_last_error", "vqemps_set_circuit",
    "vqemps_num_params", "vqemps_bond_dims", "vqemps_set_hamiltonian",
    "vqemps_free_hamiltonian", "vqemps_energy_batch", "vqemps_energy_batch_host",
    "vqemps_batch_status", "vqemps_energy_grad_batch", "vqemps_sample",
    "vqemps_sampled_energy", "vqemps_copy_sites", "vqemps_plan_stats", "vqemps_profile_energy",
    "vqemps_energy_noalloc", "vqemps_set_level_variant", "vqemps_level_variant",
    "vqemps_set_grad_checkpoint", "vqemps_set_grad_variant", "vqemps_set_split_mode", "vqemps_set_evolve_mode",
    "vqemps_set_partitions", "vqemps_free_partitions",
    "vqemps_partition_info", "vqemps_partition_bond_dims", "vqemps_partition_energy",
    "vqemps_partition_sample", "vqemps_partition_sampled_energy",
    "vqemps_mpnn_create", "vqemps_mpnn_destroy", "vqemps_mpnn_last_error", "vqemps_mpnn_num_params",
    "vqemps_mpnn_set_params", "vqemps_mpnn_get_params", "vqemps_mpnn_forward", "vqemps_mpnn_loss",
    "vqemps_mpnn_backward", "vqemps_mpnn_adam_step",
)


class VqempsOp(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("q0", ctypes.c_int32), ("q1", ctypes.c_int32),
                ("param", ctypes.c_int32), ("angle", ctypes.c_double),
                ("matrix", ctypes.c_int32), ("pad", ctypes.c_int32)]


class VqempsGraph(ctypes.Structure):
    _fields_ = [("num_nodes", ctypes.c_int32), ("num_edges", ctypes.c_int32),
                ("node_feat", ctypes.c_void_p), ("edge_feat", ctypes.c_void_p),
                ("edge_src", ctypes.c_void_p), ("edge_dst", ctypes.c_void_p),
                ("dst_off", ctypes.c_void_p), ("src_perm", ctypes.c_void_p), ("src_off", ctypes.c_void_p)]


class EngineError(RuntimeError):
    """A failing engine call; ``code`` is the vqemps_status value."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


_lib = None


def load():
    """Load the engine library once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("VQEMPS_LIBRARY", LIB_PATH))
    if not path.exists():
        raise ImportError(f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = ctypes.CDLL(str(path))
    P, I, D, V = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    u64 = ctypes.c_uint64
    sig = {
        "vqemps_create": (I, [I, I, D, D, ctypes.POINTER(P)]),
        "vqemps_destroy": (I, [P]),
        "vqemps_last_error": (ctypes.c_char_p, [P]),
        "vqemps_set_circuit": (I, [P, I, ctypes.POINTER(VqempsOp), I, ctypes.POINTER(D), I, I, I]),
        "vqemps_num_params": (I, [P, ctypes.POINTER(I)]),
        "vqemps_bond_dims": (I, [P, ctypes.POINTER(I)]),
        "vqemps_set_hamiltonian": (I, [P, ctypes.c_char_p, ctypes.POINTER(D), I, ctypes.POINTER(I)]),
        "vqemps_free_hamiltonian": (I, [P, I]),
        "vqemps_energy_batch": (I, [P, I, V, I, V, V, V]),
        "vqemps_energy_batch_host": (I, [P, I, V, I, V, V, V]),
        "vqemps_batch_status": (I, [P, ctypes.POINTER(ctypes.c_int32), I, V]),
        "vqemps_energy_grad_batch": (I, [P, I, V, I, V, V, V]),
        "vqemps_sample": (I, [P, V, I, I, u64, I, V, V]),
        "vqemps_sampled_energy": (I, [P, I, V, I, I, u64, I, I, V, V, V]),
        "vqemps_copy_sites": (I, [P, I, ctypes.POINTER(D), V]),
        "vqemps_plan_stats": (I, [P, I, ctypes.POINTER(D)]),
        "vqemps_profile_energy": (I, [P, I, V, I, ctypes.POINTER(D), ctypes.POINTER(I), V]),
        "vqemps_energy_noalloc": (I, [P, I, V, V, V, V, V]),
        "vqemps_set_level_variant": (I, [P, I]),
        "vqemps_set_grad_checkpoint": (I, [P, I]),
        "vqemps_set_grad_variant": (I, [P, I]),
        "vqemps_set_split_mode": (I, [P, I]),
        "vqemps_set_evolve_mode": (I, [P, I]),
        "vqemps_level_variant": (I, [P, I, I, ctypes.POINTER(I)]),
        "vqemps_set_partitions": (I, [P, I, V, ctypes.POINTER(VqempsOp), V, V, V, ctypes.c_char_p, V, V,
                                      I, I, ctypes.POINTER(I)]),
        "vqemps_free_partitions": (I, [P, I]),
        "vqemps_partition_info": (I, [P, I, V, V, V]),
        "vqemps_partition_bond_dims": (I, [P, I, I, ctypes.POINTER(I)]),
        "vqemps_partition_energy": (I, [P, I, V, I, V, V, V]),
        "vqemps_partition_sample": (I, [P, I, V, I, I, u64, I, V, V]),
        "vqemps_partition_sampled_energy": (I, [P, I, V, I, I, u64, I, V, V, V, V]),
        "vqemps_mpnn_create": (I, [I, I, I, I, I, I, ctypes.POINTER(P)]),
        "vqemps_mpnn_destroy": (I, [P]),
        "vqemps_mpnn_last_error": (ctypes.c_char_p, [P]),
        "vqemps_mpnn_num_params": (I, [P, ctypes.POINTER(ctypes.c_int64)]),
        "vqemps_mpnn_set_params": (I, [P, ctypes.POINTER(ctypes.c_float), ctypes.c_int64]),
        "vqemps_mpnn_get_params": (I, [P, ctypes.POINTER(ctypes.c_float), ctypes.c_int64]),
        "vqemps_mpnn_forward": (I, [P, ctypes.POINTER(VqempsGraph), V, V]),
        "vqemps_mpnn_loss": (I, [P, V, V, V, V, V]),
        "vqemps_mpnn_backward": (I, [P, ctypes.POINTER(VqempsGraph), V, V, V]),
        "vqemps_mpnn_adam_step": (I, [P, V, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                      ctypes.c_float, V]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(ctx, code: int, what: str):
    """Raise EngineError with the engine's message for a nonzero status."""
    if code == OK:
        return
    msg = load().vqemps_last_error(ctx).decode() if ctx else "invalid call"
    raise EngineError(code, f"{what}: {msg or 'status ' + str(code)}")
