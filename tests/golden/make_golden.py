"""Generate golden vectors from the reference's own CPU implementation.

Runs hp-cyber/Graph-VQE's ``ReverseMPS`` (test/tools/reverse_mps.py, imported
read-only from the reference checkout given by REFERENCE_ROOT, default
/root/reference) with torch on the CPU, and writes energies and gradients of a
set of seeded cases to ``reverse_mps_golden.json`` next to this script. The
reference checkout does not exist where the GPU tests run, so the vectors are
committed and this script is only rerun by hand.

Usage: python tests/golden/make_golden.py            (small cases, words inline)
       python tests/golden/make_golden.py --large    (benchmark-size cases)

``--large`` writes ``large_workloads_golden.json``: the reference's energies for
four parameter sets of the 40-qubit / 5,000-term / B = 256 benchmark batch
(``vqemps.workloads.batched_40q(seed=0)``) and energy plus full gradient for two
parameter sets of the 64-qubit / 20,000-term gradient workload
(``vqemps.workloads.gradient_64q(seed=0)``). Those Hamiltonians are too large to
store inline; the file records the generator call and a SHA-256 digest of the
words and coefficients, which the tests and the benchmark check before they
compare.
"""
from __future__ import annotations

import json
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
REFERENCE_ROOT = Path(os.environ.get("REFERENCE_ROOT", "/root/reference"))
sys.path.insert(0, str(REFERENCE_ROOT / "test" / "tools"))
sys.path.insert(0, str(REPO))

from reverse_mps import ReverseMPS, register, _REGISTRY  # noqa: E402  (reference code)
from oracle.workloads import random_hamiltonian  # noqa: E402


def registered_spec(n, reps, gates, pattern, initial=None):
    """Build the op spec through the reference's own ``register``."""
    k = object()
    order = [(f"t{layer}_{q}_{g}", q, layer, g)
             for layer in range(reps + 1) for q in range(n) for g in range(len(gates))]
    pairs = []
    for _ in range(reps):
        edges = [(i, i + 1) for i in range(n - 1)]
        if pattern == "reverse_linear":
            edges.reverse()
        pairs.append(edges)
    register(k, n, reps, gates, pattern, initial, order, pairs, True)
    spec = _REGISTRY.pop(id(k))[1]
    return spec


def case(name, spec, words, coeffs, x, grad=True):
    p = ReverseMPS(spec, words, coeffs, device="cpu")
    if grad:
        e, g = p.value_gradient(np.asarray(x))
        g = [float(v) for v in g]
    else:
        import torch
        with torch.no_grad():
            sites = p.sites(torch.tensor(np.asarray(x), dtype=torch.float64))
            e = 0.0
            for i in range(0, len(words), p.chunk):
                e += float(p.energy_chunk(sites, words[i:i + p.chunk], p.coeffs[i:i + p.chunk]))
        g = None
    return dict(name=name, spec=dict(n=spec["n"], ops=[list(o) for o in spec["ops"]],
                                     initial=spec.get("initial"), count=spec["count"]),
                words=list(words), coeffs=[float(c) for c in coeffs], x=[float(v) for v in x],
                energy=float(e), gradient=g)


def main():
    out = []
    # the reference's own unit-test circuit (test/tests/test_reverse_mps.py:47-53)
    spec = dict(n=3, initial="+", count=4,
                ops=[("ry", 0, 0), ("rz", 1, 1), ("cx", 0, 1), ("rx", 2, 2), ("cx", 1, 2), ("ry", 1, 3)])
    out.append(case("unit_test_circuit", spec, ["YXI", "ZZI", "III", "XXZ"], [.3, -.7, .4, .2],
                    [.2, -.4, .8, .1]))
    rng = np.random.default_rng(2024)
    for n, reps, gates, pattern, terms, wmax, zf in [
        (3, 2, ("ry", "rz"), "linear", 6, 3, 0.5),
        (3, 2, ("ry", "rz"), "reverse_linear", 6, 3, 0.5),
        (6, 3, ("ry",), "linear", 40, 4, 0.9),
        (6, 3, ("ry", "rz"), "reverse_linear", 40, 4, 0.5),
        (12, 4, ("ry",), "linear", 300, 4, 0.9),
        (12, 4, ("ry",), "reverse_linear", 300, 4, 0.9),
        (9, 2, ("rx", "rz"), "linear", 60, 5, 0.3),
    ]:
        spec = registered_spec(n, reps, gates, pattern)
        words, coeffs = random_hamiltonian(rng, n, terms, wmax, zf)
        x = rng.uniform(-np.pi, np.pi, spec["count"])
        out.append(case(f"{pattern}_{n}q_{reps}l_{'_'.join(gates)}", spec, words, coeffs, x))
    # 40-qubit reverse_linear RY ansatz, 5,000 terms: energies only (two parameter sets)
    spec = registered_spec(40, 4, ("ry",), "reverse_linear")
    words, coeffs = random_hamiltonian(np.random.default_rng(7), 40, 5000, 6)
    for k in range(2):
        x = np.random.default_rng(100 + k).uniform(-np.pi, np.pi, spec["count"])
        out.append(case(f"reverse_linear_40q_5000t_{k}", spec, words, coeffs, x, grad=False))
    (HERE / "reverse_mps_golden.json").write_text(json.dumps(out))
    print(f"wrote {len(out)} cases")


def _check_spec(name, spec, n, pattern):
    ref = registered_spec(n, 4, ("ry",), pattern)
    ours = [tuple(o) for o in spec["ops"]]
    assert ours == [tuple(o) for o in ref["ops"]] and spec["count"] == ref["count"], name
    return ref


def main_large():
    sys.path.insert(0, str(REPO / "graph-vqe_b200"))
    from vqemps import workloads as VW  # the generators bench.py and the tests use
    workload_digest = VW.workload_digest
    import torch
    torch.set_num_threads(os.cpu_count() or 1)
    out = {}
    # the benchmark batch: 40 qubits, reverse_linear, 5,000 terms, 256 SPSA probes
    spec, words, coeffs, thetas = VW.batched_40q(seed=0, batch=256)
    ref = _check_spec("batched_40q", spec, 40, "reverse_linear")
    idx = [0, 1, 128, 255]
    cases = []
    for i in idx:
        t0 = time.time()
        c = case(f"batched_40q_{i}", ref, words, coeffs, thetas[i], grad=False)
        cases.append(c["energy"])
        print(f"batched_40q[{i}] E = {c['energy']!r} ({time.time() - t0:.1f} s)", flush=True)
    out["batched_40q"] = dict(call="vqemps.workloads.batched_40q(seed=0, batch=256)", n=40, terms=len(words),
                              digest=workload_digest(words, coeffs), indices=idx, energies=cases)
    # the gradient workload: 64 qubits, linear, 20,000 terms, 32 parameter sets
    spec, words, coeffs, thetas = VW.gradient_64q(seed=0, batch=32)
    ref = _check_spec("gradient_64q", spec, 64, "linear")
    idx = [0, 17]
    es, gs = [], []
    for i in idx:
        t0 = time.time()
        c = case(f"gradient_64q_{i}", ref, words, coeffs, thetas[i], grad=True)
        es.append(c["energy"])
        gs.append(c["gradient"])
        print(f"gradient_64q[{i}] E = {c['energy']!r} ({time.time() - t0:.1f} s)", flush=True)
    out["gradient_64q"] = dict(call="vqemps.workloads.gradient_64q(seed=0, batch=32)", n=64, terms=len(words),
                               digest=workload_digest(words, coeffs), indices=idx, energies=es, gradients=gs)
    (HERE / "large_workloads_golden.json").write_text(json.dumps(out))
    print("wrote large_workloads_golden.json")


if __name__ == "__main__":
    if "--large" in sys.argv:
        main_large()
    else:
        main()
