"""Hamiltonian ingest and readout order against the reference's converter
(cudaq.py:25-47) and decoder (readout.py:4-9), via the golden outputs of
tests/golden/make_ingest_golden.py; and the partition plan of the strategy
against the blocks the reference's own strategy code chose
(tests/golden/strategy_golden.json)."""
import json
from pathlib import Path

import numpy as np
import pytest

from vqemps import ingest

G = json.loads((Path(__file__).parent / "golden" / "ingest_golden.json").read_text())
S = json.loads((Path(__file__).parent / "golden" / "strategy_golden.json").read_text())


class ListOp:
    def __init__(self, pairs):
        self.pairs = pairs

    def to_list(self):
        return self.pairs


def _nonzero(words, coeffs):
    return {w: c for w, c in zip(words, coeffs) if c != 0.0}


@pytest.mark.parametrize("case", G["converter"], ids=lambda c: f"{len(c['pairs'])}terms_rev{c['reverse']}")
def test_converter_equals_reference(case):
    """The reference's operator starts from the scalar 0.0 (cudaq.py:31), which the
    spin algebra keeps as an identity term with coefficient 0; terms with a zero
    coefficient add nothing and are left out of the comparison."""
    pairs = [(lab, complex(re, im)) for lab, (re, im) in case["pairs"]]
    ref = _nonzero(case["words"], case["coeffs"])
    words, coeffs = ingest.sparse_pauli_terms(ListOp(pairs), reverse_qubit_order=case["reverse"])
    assert _nonzero(words, coeffs.tolist()) == ref
    spin = ingest.sparse_pauli_to_spin(pairs, reverse_qubit_order=case["reverse"])
    ws, cs = spin.words(len(pairs[0][0]))
    assert _nonzero(ws, [float(np.real(c)) for c in cs]) == ref


def test_converter_rejects_bad_labels():
    with pytest.raises(ValueError):
        ingest.sparse_pauli_terms([("ZQ", 1.0)])


@pytest.mark.parametrize("case", G["readout"], ids=lambda c: str(len(c["counts"])))
def test_readout_equals_reference(case):
    assert ingest.protein_probabilities(case["counts"]) == case["probabilities"]
    with pytest.raises(ValueError):
        ingest.protein_probabilities({})


def test_partition_plan_equals_reference_blocks():
    from vqemps import workloads as VW
    from vqemps.strategy import PartitionPlan
    words, coeffs = VW.random_hamiltonian(np.random.default_rng(S["hamiltonian_seed"]), S["n"], S["terms"], S["wmax"])
    assert VW.workload_digest(words, coeffs) == S["digest"]
    plan = PartitionPlan(S["n"], words, coeffs, reps=S["reps"], su2_gates=tuple(S["su2_gates"]),
                         entanglement=S["entanglement"], max_block_qubits=S["max_block_qubits"], seed=S["seed"])
    assert plan.blocks == S["blocks"]
    # the same Hamiltonian given as qiskit labels (q0 rightmost) through the converter
    w2, c2 = ingest.sparse_pauli_terms([(w[::-1], c) for w, c in zip(words, coeffs)])
    plan2 = PartitionPlan(S["n"], w2, c2, reps=S["reps"], su2_gates=tuple(S["su2_gates"]),
                          entanglement=S["entanglement"], max_block_qubits=S["max_block_qubits"], seed=S["seed"])
    assert plan2.blocks == S["blocks"]
