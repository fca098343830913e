"""Hamiltonian ingest and readout conventions at the boundary.

* ``sparse_pauli_terms`` / ``sparse_pauli_to_spin``: a qiskit ``SparsePauliOp``
  (anything with ``to_list()``) or a plain list of (label, coefficient) pairs
  to the engine's qubit-indexed words, as the reference's
  ``qiskit_sparsepauliop_to_cudaq_spin`` does it
  (test/sources/independent-vqe/Qiskit_VQE/cudaq.py:25-47): a label's rightmost
  character is qubit 0 (``reverse_qubit_order=True``), terms with a zero
  coefficient are skipped, the real part of each coefficient is kept, and
  equal words add up.
* ``protein_probabilities``: sample counts (qubit 0 leftmost, the engine's and
  CUDA-Q's key order) to the protein decoder's probabilities (qubit 0
  rightmost), test/tools/readout.py:4-9.
"""
from __future__ import annotations

import numpy as np


def _pairs(op):
    return op.to_list() if hasattr(op, "to_list") else list(op)


def sparse_pauli_terms(op, reverse_qubit_order: bool = True):
    """(words, coeffs): words indexed by qubit (word[q] acts on qubit q), ready for
    ``Engine.set_hamiltonian``; equal words merged in order of first occurrence."""
    index, words, coeffs = {}, [], []
    for label, coeff in _pairs(op):
        if coeff == 0:
            continue
        label = str(label)
        n = len(label)
        chars = ["I"] * n
        for idx, ch in enumerate(label):
            if ch not in "IXYZ":
                raise ValueError(f"invalid Pauli label {label!r}")
            chars[(n - 1 - idx) if reverse_qubit_order else idx] = ch
        word = "".join(chars)
        c = float(np.real(coeff))
        if word in index:
            coeffs[index[word]] += c
        else:
            index[word] = len(words)
            words.append(word)
            coeffs.append(c)
    return words, np.asarray(coeffs, dtype=float)


def sparse_pauli_to_spin(op, reverse_qubit_order: bool = True):
    """The same terms as a ``vqemps.shim`` spin operator (the object ``observe`` takes)."""
    from .shim import SpinOperator, Term  # noqa: F401
    from .shim import spin
    words, coeffs = sparse_pauli_terms(op, reverse_qubit_order)
    total = None
    for w, c in zip(words, coeffs):
        term = None
        for q, ch in enumerate(w):
            if ch == "I":
                continue
            f = {"X": spin.x, "Y": spin.y, "Z": spin.z}[ch](q)
            term = f if term is None else term * f
        term = c * (term if term is not None else spin.i(0))
        total = term if total is None else total + term
    return total if total is not None else 0.0 * spin.i(0)


def protein_probabilities(counts):
    """Counts keyed q0-left to probabilities keyed q0-right (readout.py:4-9)."""
    total = sum(counts.values())
    if total <= 0:
        raise ValueError("Cannot decode an empty measurement histogram")
    return {bits[::-1]: count / total for bits, count in counts.items()}
