"""Timed CPU baseline -- TEST INFRASTRUCTURE (bench.py's cpu_baseline / reference arm).

Times the C restatement of the reference's CPU energy path (ReverseMPS on the
exact bond-doubling MPS, 128-term chunks; oracle/cpu_energy.c) on the 40-qubit,
5,000-term workload, one parameter set after another, for a bounded time.
"""
from __future__ import annotations

import ctypes
import os
import time

import numpy as np

from . import cbuild
from .mps_oracle import bond_doubling_sites
from .workloads import batched_40q

_lib = None


def load():
    global _lib
    if _lib is None:
        path = cbuild.build()
        lib = ctypes.CDLL(str(path))
        lib.cpu_energy.restype = ctypes.c_double
        lib.cpu_energy.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                                   ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int]
        _lib = lib
    return _lib


def padded(sites):
    n = len(sites)
    out = np.zeros((n, 16, 2, 16), dtype=np.complex128)
    dims = [1] * (n + 1)
    for q, a in enumerate(sites):
        out[q, :a.shape[0], :, :a.shape[2]] = a
        dims[q] = a.shape[0]
        dims[q + 1] = a.shape[2]
    return out, np.asarray(dims, dtype=np.int32)


def energy(spec, words, coeffs, x, threads=None, chunk=128):
    """ReverseMPS energy on the CPU (bond-doubling sites + chunked prefix sweep)."""
    lib = load()
    sites, dims = padded(bond_doubling_sites(spec, x))
    buf = np.ascontiguousarray(sites).view(np.float64)
    coeffs = np.ascontiguousarray(coeffs, dtype=np.float64)
    return lib.cpu_energy(spec["n"], buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                          dims.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), "".join(words).encode(),
                          coeffs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(words), chunk,
                          threads or os.cpu_count() or 1)


class Workload:
    """The 40-qubit, 5,000-term workload, built once."""

    def __init__(self, batch: int = 256):
        self.spec, self.words, self.coeffs, self.thetas = batched_40q(seed=0, batch=batch)
        self.next = 0

    def run(self, count: int, threads: int) -> float:
        """Evaluate ``count`` parameter sets one after another; returns seconds."""
        t0 = time.perf_counter()
        for _ in range(count):
            energy(self.spec, self.words, self.coeffs, self.thetas[self.next % len(self.thetas)], threads)
            self.next += 1
        return time.perf_counter() - t0


def describe(k, dt, threads):
    return (f"{k} of the 256 parameter sets evaluated one after another in {dt:.1f} s "
            f"(C/OpenMP restatement of ReverseMPS energy, 128-term chunks, {threads} threads)")


def energy_rate(seconds: float, threads: int, batch: int = 256):
    w = Workload(batch)
    w.run(1, threads)                                        # warm-up (load, page in)
    t0 = time.perf_counter()
    k = 0
    while True:
        w.run(1, threads)
        k += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return dict(value=k / dt, evals=k, seconds=dt, threads=threads, sample=describe(k, dt, threads))
