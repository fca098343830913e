"""Golden outputs of the reference's Hamiltonian converter and readout decoder.

Extracts ``qiskit_sparsepauliop_to_cudaq_spin`` from
test/sources/independent-vqe/Qiskit_VQE/cudaq.py by AST (the module itself
imports CUDA-Q and qiskit, absent here), runs it with ``vqemps.shim.spin`` as the
spin-operator algebra on lists of (label, coefficient) pairs standing in for
``SparsePauliOp.to_list()``, and records the resulting operator's qubit-indexed
words and coefficients; runs test/tools/readout.py's ``protein_probabilities``
on sample counts. Writes ``ingest_golden.json``.

Usage: python tests/golden/make_ingest_golden.py
"""
from __future__ import annotations

import ast
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
REFERENCE_ROOT = Path(os.environ.get("REFERENCE_ROOT", "/root/reference"))
sys.path.insert(0, str(REPO / "graph-vqe_b200"))
sys.path.insert(0, str(REFERENCE_ROOT / "test" / "tools"))

from readout import protein_probabilities  # noqa: E402  (reference code)
from vqemps import shim  # noqa: E402


class ListOp:
    def __init__(self, pairs):
        self.pairs = pairs
        self.num_qubits = len(pairs[0][0])

    def to_list(self):
        return self.pairs


def converter():
    path = REFERENCE_ROOT / "test" / "sources" / "independent-vqe" / "Qiskit_VQE" / "cudaq.py"
    tree = ast.parse(path.read_text())
    fn = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "qiskit_sparsepauliop_to_cudaq_spin")
    ns = dict(spin=shim.spin, SparsePauliOp=object)
    exec(compile(ast.fix_missing_locations(ast.Module(body=[fn], type_ignores=[])), str(path), "exec"), ns)
    return ns["qiskit_sparsepauliop_to_cudaq_spin"]


def main():
    convert = converter()
    rng = np.random.default_rng(5)
    cases = [
        [("ZIXY", 1.5), ("IIII", 0.0), ("ZIXY", 0.5 + 0.0j), ("XXII", -2.0), ("IIIZ", 0.25 + 1e-14j)],
        [("YYZZX", 0.7), ("IIIII", 3.0), ("ZIIIZ", -1.25), ("XIYIZ", 0.0)],
    ]
    labels = ["".join(rng.choice(list("IXYZ"), 9)) for _ in range(40)]
    cases.append([(lab, complex(rng.normal(), 0.0)) for lab in labels])
    out = dict(converter=[], readout=[])
    for pairs in cases:
        for reverse in (True, False):
            H = convert(ListOp(pairs), reverse_qubit_order=reverse)
            width = len(pairs[0][0])
            ws, cs = H.words(width)
            out["converter"].append(dict(pairs=[[lab, [float(np.real(c)), float(np.imag(c))]] for lab, c in pairs],
                                         reverse=reverse, words=ws, coeffs=[float(np.real(c)) for c in cs]))
    for counts in ({"1000000": 1000}, {"1010000": 750, "0100001": 250},
                   {"0000000": 600, "1111111": 300, "1000000": 100}):
        out["readout"].append(dict(counts=counts, probabilities=protein_probabilities(counts)))
    (HERE / "ingest_golden.json").write_text(json.dumps(out))
    print(f"wrote {len(out['converter'])} converter and {len(out['readout'])} readout cases")


if __name__ == "__main__":
    main()
