"""Generate a golden run of the reference's own partition warm start.

The reference's strategy class (IndependentSubspaceVQE in
test/sources/independent-vqe/Qiskit_VQE/independent_vqe.py) cannot be imported
here: its module imports CUDA-Q and qiskit. As the reference's own tests do
(test/tests/test_single_pass.py:12-22, test_global_ansatz.py:12-27), this script
extracts the production class from the source by AST -- its constructor,
_partition, _build_kernel, _spin, _run_vqe, _remember_global and
_minimize_model, unchanged -- together with qiskit_sparsepauliop_to_cudaq_spin
(cudaq.py), pairs_for_pattern (efficientsu2.py) and configure_full_bond
(mps_config.py), and runs it with:

* ``vqemps.shim`` standing in for the ``cudaq`` module (kernel building and
  spin-operator algebra are pure Python there);
* a small stand-in for qiskit's ``SparsePauliOp`` (labels with q0 rightmost,
  ``simplify`` merging identical labels in order of first occurrence and
  dropping exact zeros, the restatement the oracle also uses);
* a stand-in for the SubspaceVQE base class that sets the constructor's
  attributes and evaluates ``_evaluate_energy`` with the oracle's exact
  energy (pinned to the reference's ReverseMPS to 1e-9) of the recorded kernel.

It records the blocks, every local solve's best energy, the assembled warm
start and its energy, the global solve and the best energy, for one seeded
16-qubit Hamiltonian, in ``strategy_golden.json``. The GPU test runs
``vqemps.strategy.IndependentPartitionVQE`` on the same inputs and compares.

Usage: python tests/golden/make_strategy_golden.py
"""
from __future__ import annotations

import ast
import importlib.util
import json
import os
import sys
import time
from concurrent.futures import ThreadPoolExecutor
from contextlib import nullcontext
from itertools import combinations
from pathlib import Path
from types import SimpleNamespace
from typing import Callable, Iterable, List, Sequence, Tuple, Union

import networkx as nx
import numpy as np
from scipy.optimize import minimize

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
REFERENCE_ROOT = Path(os.environ.get("REFERENCE_ROOT", "/root/reference"))
SRC = REFERENCE_ROOT / "test" / "sources" / "independent-vqe" / "Qiskit_VQE"
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "graph-vqe_b200"))

from oracle import mps_oracle as O  # noqa: E402
from vqemps import shim  # noqa: E402
from vqemps import workloads as VW  # noqa: E402

N, TERMS, WMAX, SEED, HSEED = 16, 240, 4, 3, 21


class SparsePauliOpStandIn:
    """The part of qiskit's SparsePauliOp the strategy uses (labels: q0 rightmost)."""

    def __init__(self, labels, coeffs):
        self.labels = list(labels)
        self.coeffs = np.asarray(coeffs, dtype=complex)
        self.num_qubits = len(self.labels[0])

    @classmethod
    def from_list(cls, terms):
        return cls([t[0] for t in terms], [t[1] for t in terms])

    def to_list(self):
        return list(zip(self.labels, self.coeffs))

    def simplify(self, atol=None, rtol=None):
        index, labels, coeffs = {}, [], []
        for lab, c in zip(self.labels, self.coeffs):
            if lab in index:
                coeffs[index[lab]] += c
            else:
                index[lab] = len(labels)
                labels.append(lab)
                coeffs.append(c)
        keep = [i for i, c in enumerate(coeffs) if c != 0]
        if not keep:
            return SparsePauliOpStandIn(["I" * self.num_qubits], [0.0])
        return SparsePauliOpStandIn([labels[i] for i in keep], [coeffs[i] for i in keep])


class SubspaceVQEStandIn:
    """Attributes of SubspaceVQE.__init__ (subspace_vqe.py:53-200) the strategy reads."""

    class EarlyStop(Exception):
        pass

    def __init__(self, hamiltonian=None, num_qubits=0, shots=8192, max_epochs=3, window_size=2, block_maxiter=30,
                 global_refinement=True, global_maxiter=10, reps=4, entanglement="circular", su2_gates=("ry", "rz"),
                 energy_tol=1e-4, seed=0, use_gradient_optimizer=False, **_):
        self.hamiltonian = hamiltonian
        self.num_qubits = int(num_qubits)
        self.shots = int(shots)
        self.max_epochs = int(max_epochs)
        self.block_maxiter = int(block_maxiter)
        self.global_refinement = bool(global_refinement)
        self.global_maxiter = int(global_maxiter)
        self.reps = int(reps)
        self.entanglement = entanglement
        self.su2_gates = tuple(su2_gates)
        self.energy_tol = float(energy_tol)
        self.seed = seed
        self.use_gradient_optimizer = use_gradient_optimizer
        self.num_parallel_workers = 1
        self.num_gpus_detected = 1
        self.nfev = 0
        self._evaluation_seconds = 0.0
        self.recorded = []

    def _timed_optimizer(self, *args, **kwargs):
        return nullcontext()

    def _record_iteration(self, energy, status="accepted"):
        self.recorded.append((float(energy), status))

    def _evaluate_energy(self, x, qpu_id=None, kernel=None, hamiltonian=None, **_):
        kernel = self.kernel if kernel is None else kernel
        hamiltonian = self.hamiltonian if hamiltonian is None else hamiltonian
        self.nfev += 1
        ops, _, _ = kernel.program()
        ang = kernel.angles(np.asarray(x, dtype=float))[0]
        width = max(2, kernel.width)
        words, coeffs = hamiltonian.words(width)
        spec = dict(n=width, ops=[tuple(o) for o in ops], initial=None, count=len(ang))
        return float(O.reverse_energy(spec, words, np.real(np.asarray(coeffs, dtype=complex)), ang))


def extract(path, names, namespace, class_name=None):
    tree = ast.parse(Path(path).read_text())
    body = []
    for node in tree.body:
        if class_name is not None and isinstance(node, ast.ClassDef) and node.name == class_name:
            body.append(node)
        elif isinstance(node, ast.FunctionDef) and node.name in names:
            body.append(node)
    module = ast.Module(body=[ast.ImportFrom(module="__future__", names=[ast.alias(name="annotations")], level=0)]
                        + body, type_ignores=[])
    exec(compile(ast.fix_missing_locations(module), str(path), "exec"), namespace)
    return namespace


def main():
    ns = dict(np=np, nx=nx, time=time, minimize=minimize, combinations=combinations,
              ThreadPoolExecutor=ThreadPoolExecutor, Callable=Callable, Iterable=Iterable, List=List,
              Sequence=Sequence, Tuple=Tuple, Union=Union, pi=np.pi)
    cudaq_stand_in = SimpleNamespace(make_kernel=shim.make_kernel, spin=shim.spin)
    ns.update(cudaq=cudaq_stand_in, spin=shim.spin, SparsePauliOp=SparsePauliOpStandIn,
              SubspaceVQE=SubspaceVQEStandIn)
    extract(SRC / "cudaq.py", {"qiskit_sparsepauliop_to_cudaq_spin"}, ns)
    extract(SRC / "efficientsu2.py", {"pairs_for_pattern"}, ns)
    spec = importlib.util.spec_from_file_location("reference_mps_config", SRC / "mps_config.py")
    mps_config = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mps_config)
    ns.update(configure_full_bond=mps_config.configure_full_bond, configure_gpu_groups=lambda *a, **k: "")
    extract(SRC / "independent_vqe.py", set(), ns, class_name="IndependentSubspaceVQE")
    Strategy = ns["IndependentSubspaceVQE"]

    rng = np.random.default_rng(HSEED)
    words, coeffs = VW.random_hamiltonian(rng, N, TERMS, WMAX)          # qubit-indexed words
    labels = [w[::-1] for w in words]                                    # qiskit labels: q0 rightmost
    op = SparsePauliOpStandIn(labels, coeffs)
    solver = Strategy(qiskit_hamiltonian=op, hamiltonian=None, num_qubits=N, reps=4, su2_gates=("ry",),
                      entanglement="linear", max_block_qubits=12, energy_tol=1.0, block_maxiter=30,
                      global_maxiter=10, seed=SEED, use_gradient_optimizer=True, shots=-1)
    t0 = time.time()
    history, best_params, _, results = solver._run_vqe()
    out = dict(n=N, terms=TERMS, wmax=WMAX, hamiltonian_seed=HSEED, seed=SEED, reps=4, su2_gates=["ry"],
               entanglement="linear", max_block_qubits=12, energy_tol=1.0, block_maxiter=30, global_maxiter=10,
               use_gradient_optimizer=True,
               digest=VW.workload_digest(words, coeffs),
               blocks=solver.blocks,
               local_energies=[float(r["energy"]) for r in solver.local_results],
               local_accepted=[int(r["accepted_iterations"]) for r in solver.local_results],
               local_stop=[str(r["stop_reason"]) for r in solver.local_results],
               warm_start_params=[float(v) for v in solver.warm_start_params],
               warm_start_energy=float(solver.warm_start_energy),
               global_energy=float(solver.global_results[0]["energy"]) if solver.global_results else None,
               global_accepted=int(solver.global_results[0]["accepted_iterations"]) if solver.global_results else 0,
               global_stop=str(solver.global_results[0]["stop_reason"]) if solver.global_results else None,
               best_energy=float(results[0][0]), best_params=[float(v) for v in best_params],
               energy_evaluations=solver.nfev)
    (HERE / "strategy_golden.json").write_text(json.dumps(out))
    print(json.dumps({k: v for k, v in out.items() if "params" not in k}), f"({time.time() - t0:.0f} s)")


if __name__ == "__main__":
    main()
