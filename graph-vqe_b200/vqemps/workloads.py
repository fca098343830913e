"""Seeded synthetic workloads of the benchmarks and the warm-start training set.

The reference's protein Hamiltonians (Z/I-only lattice operators,
Protein_Folding/peptide/pauli_ops_builder.py:25-50) need qiskit to be
generated, so seeded synthetic Pauli sums with the benchmark sizes stand in:

* a term draws weight w ~ U{1..wmax} on distinct random qubits; with p = 0.9 it
  is a Z-string, otherwise each support qubit is U{X, Y, Z};
* coefficients are FP64: N(0, 1) with p = 0.8, +-U(100, 1000) with p = 0.2;
* angles are U(-pi, pi).

Words are strings over I/X/Y/Z indexed by qubit. Circuits are spec dicts
``{n, ops, initial, count}`` of the hardware-efficient RY ansatz.
"""
from __future__ import annotations

import hashlib

import numpy as np

from .strategy import ansatz_ops


def ansatz_spec(n: int, reps: int = 4, gates=("ry",), pattern: str = "linear"):
    ops, count = ansatz_ops(n, reps, tuple(gates), pattern)
    return dict(n=n, ops=ops, initial=None, count=count)


def random_hamiltonian(rng: np.random.Generator, n: int, terms: int, wmax: int, z_fraction: float = 0.9):
    words, coeffs = [], []
    for _ in range(terms):
        w = int(rng.integers(1, min(wmax, n) + 1))
        support = rng.choice(n, size=w, replace=False)
        chars = ["I"] * n
        z_only = rng.random() < z_fraction
        for q in support:
            chars[int(q)] = "Z" if z_only else "XYZ"[int(rng.integers(0, 3))]
        words.append("".join(chars))
        if rng.random() < 0.8:
            coeffs.append(float(rng.normal()))
        else:
            sign = 1.0 if rng.random() < 0.5 else -1.0
            coeffs.append(sign * float(rng.uniform(100.0, 1000.0)))
    return words, np.asarray(coeffs, dtype=np.float64)


def workload_digest(words, coeffs) -> str:
    """SHA-256 of a Hamiltonian: the words newline-joined in ASCII, then the
    coefficients as little-endian FP64. Pins a regenerated workload to recorded
    values without storing its terms."""
    h = hashlib.sha256("\n".join(words).encode("ascii"))
    h.update(np.ascontiguousarray(coeffs, dtype="<f8").tobytes())
    return h.hexdigest()


def plain_12q(seed: int = 0):
    """12 qubits, linear RY ansatz, 4 layers + final RY (60 angles), 300 terms, wmax 4."""
    rng = np.random.default_rng(seed)
    spec = ansatz_spec(12, 4, ("ry",), "linear")
    words, coeffs = random_hamiltonian(rng, 12, 300, 4)
    return spec, words, coeffs, rng.uniform(-np.pi, np.pi, spec["count"])


def spsa_probes(rng: np.random.Generator, center: np.ndarray, pairs: int, c: float):
    """SPSA +-c Rademacher probe pairs (spsa_optimizer.py:59-63) as [2 * pairs, P]."""
    out = np.empty((2 * pairs, center.size))
    for k in range(pairs):
        delta = rng.choice(np.array([-1.0, 1.0]), size=center.size)
        out[2 * k] = center + c * delta
        out[2 * k + 1] = center - c * delta
    return out


def batched_40q(seed: int = 0, batch: int = 256, terms: int = 5000, n: int = 40):
    """40 qubits, reverse_linear RY ansatz (200 angles), 5,000 terms of weight <= 6,
    ``batch`` parameter sets = SPSA +-0.1 probe pairs around a seeded point."""
    rng = np.random.default_rng(seed)
    spec = ansatz_spec(n, 4, ("ry",), "reverse_linear")
    words, coeffs = random_hamiltonian(rng, n, terms, 6)
    center = rng.uniform(-np.pi, np.pi, spec["count"])
    return spec, words, coeffs, spsa_probes(rng, center, (batch + 1) // 2, 0.1)[:batch]


def uneven_partitions(seed: int = 0, partitions: int = 64, nmin: int = 8, nmax: int = 48,
                      tmin: int = 200, tmax: int = 3000):
    """Independent partitions of uneven width and term count (linear, 4 layers, wmax 4)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(partitions):
        n = int(rng.integers(nmin, nmax + 1))
        t = int(rng.integers(tmin, tmax + 1))
        spec = ansatz_spec(n, 4, ("ry",), "linear")
        words, coeffs = random_hamiltonian(rng, n, t, 4)
        out.append((spec, words, coeffs, rng.uniform(-np.pi, np.pi, spec["count"])))
    return out


def gradient_64q(seed: int = 0, batch: int = 32, terms: int = 20000, n: int = 64):
    """64 qubits, linear RY ansatz (320 angles), 20,000 terms of weight <= 6."""
    rng = np.random.default_rng(seed)
    spec = ansatz_spec(n, 4, ("ry",), "linear")
    words, coeffs = random_hamiltonian(rng, n, terms, 6)
    return spec, words, coeffs, rng.uniform(-np.pi, np.pi, (batch, spec["count"]))


def warm_start_problem(seed: int, nmin: int = 16, nmax: int = 48, terms_per_qubit: int = 25, wmax: int = 4):
    """One training Hamiltonian of the learned warm start: n ~ U{nmin..nmax},
    T = terms_per_qubit * n (the 12-qubit / 300-term ratio of the plain
    benchmark), weight <= wmax."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(nmin, nmax + 1))
    words, coeffs = random_hamiltonian(rng, n, terms_per_qubit * n, wmax)
    return n, words, coeffs


def warm_start_test_problem(seed: int, n: int = 96, terms: int = 40000, wmax: int = 4):
    """One evaluation Hamiltonian of the learned warm start (unseen width and size)."""
    rng = np.random.default_rng(seed)
    words, coeffs = random_hamiltonian(rng, n, terms, wmax)
    return n, words, coeffs
