"""GPU: the plain partition warm start with batched local solves.

The concurrent local solves (one partition-set call per round) must follow
exactly the trajectories of one-block-at-a-time solves, and the global
refinement with the adjoint gradient must match the reference's
parameter-shift refinement."""
import numpy as np
import pytest
import torch

from oracle import mps_oracle as O
from oracle.workloads import random_hamiltonian

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vq(cuda_device):
    import vqemps
    return vqemps


def _problem(n=20, T=150, seed=2):
    rng = np.random.default_rng(seed)
    words, coeffs = random_hamiltonian(rng, n, T, 4)
    return n, words, coeffs


def test_batched_local_solves_equal_sequential_solves(vq):
    from vqemps.strategy import IndependentPartitionVQE, minimize_model
    n, words, coeffs = _problem()
    eng = vq.Engine(0, 16)
    strat = IndependentPartitionVQE(eng, n, words, coeffs, block_maxiter=6, max_block_qubits=8)
    theta = strat.initial_theta()
    batched = strat.solve_locals(theta)
    assert strat.local_calls < sum(len(r["history"]) for r in batched)
    for m, r in zip(strat.local_models, batched):
        se = vq.Engine(0, 16)
        se.set_circuit(m["width"], m["ops"], site_order="msb")
        se.set_level_variant("dmma3_pf")
        se.set_split_mode("off")          # the partition set's plan
        h = se.set_hamiltonian([t for t, _ in m["terms"]], [c for _, c in m["terms"]])
        energies = lambda X: se.energy(h, torch.as_tensor(X, device=se.device)).cpu().numpy()  # noqa: E731
        seq = minimize_model(theta[m["parameter_indices"]], 6, m["constant"], energies, None,
                             energy_tol=strat.energy_tol)
        assert seq["energy"] == r["energy"]
        assert np.array_equal(seq["params"], r["params"])
        assert seq["history"] == r["history"]
        # the oracle agrees with the final local energy
        spec = dict(n=m["width"], ops=m["ops"], initial=None, count=m["count"])
        ref = O.reverse_energy(spec, [t for t, _ in m["terms"]], np.array([c for _, c in m["terms"]]), r["params"])
        assert abs(ref - r["energy"]) <= 1e-9 * max(1.0, abs(ref))


def test_global_refinement_adjoint_matches_parameter_shift(vq):
    from vqemps.strategy import IndependentPartitionVQE, minimize_model
    n, words, coeffs = _problem(n=14, T=120, seed=5)
    eng = vq.Engine(0, 16)
    strat = IndependentPartitionVQE(eng, n, words, coeffs, global_maxiter=3, energy_tol=1e-9)
    theta = strat.initial_theta()
    adj = strat.refine(theta)
    shift = minimize_model(theta, 3, False, strat.energy, None, energy_tol=strat.energy_tol)
    assert abs(adj["energy"] - shift["energy"]) <= 1e-8 * max(1.0, abs(shift["energy"]))
    assert np.allclose(adj["params"], shift["params"], atol=1e-6)


def test_full_plain_method_run(vq):
    from vqemps.strategy import IndependentPartitionVQE
    n, words, coeffs = _problem(n=24, T=200, seed=9)
    eng = vq.Engine(0, 16)
    strat = IndependentPartitionVQE(eng, n, words, coeffs, block_maxiter=10, global_maxiter=5)
    out = strat.run()
    assert np.isfinite(out["warm_start_energy"]) and out["best_energy"] <= out["warm_start_energy"]
    ref = O.reverse_energy(dict(n=n, ops=strat.problem.ops, initial=None, count=strat.num_params),
                           strat.plan.words, strat.plan.coeffs, out["best_params"])
    assert abs(ref - out["best_energy"]) <= 1e-9 * max(1.0, abs(ref))


def test_run_equals_reference_strategy_golden(vq):
    """The whole plain method against a run of the reference's own strategy code
    (tests/golden/strategy_golden.json: IndependentSubspaceVQE's constructor,
    _partition, _run_vqe and _minimize_model extracted from the source and run
    with the oracle's energies): the same blocks, local solve energies and
    iteration counts, warm start, and best energy. Energies agree to the
    engine's FP64 rounding (1e-9 relative); the optimizers see values that
    differ in the last bits, so parameters agree to 1e-6."""
    import json
    from pathlib import Path
    from vqemps import workloads as VW
    from vqemps.strategy import IndependentPartitionVQE
    g = json.loads((Path(__file__).parent / "golden" / "strategy_golden.json").read_text())
    words, coeffs = VW.random_hamiltonian(np.random.default_rng(g["hamiltonian_seed"]), g["n"], g["terms"], g["wmax"])
    assert VW.workload_digest(words, coeffs) == g["digest"]
    eng = vq.Engine(0, 16)
    strat = IndependentPartitionVQE(eng, g["n"], words, coeffs, reps=g["reps"], su2_gates=tuple(g["su2_gates"]),
                                    entanglement=g["entanglement"], max_block_qubits=g["max_block_qubits"],
                                    energy_tol=g["energy_tol"], block_maxiter=g["block_maxiter"],
                                    global_maxiter=g["global_maxiter"], use_gradient_optimizer=g["use_gradient_optimizer"],
                                    seed=g["seed"])
    out = strat.run()
    rel = lambda a, b: abs(a - b) / max(1.0, abs(b))  # noqa: E731
    assert out["blocks"] == g["blocks"]
    for r, e, acc, stop in zip(out["local_results"], g["local_energies"], g["local_accepted"], g["local_stop"]):
        assert rel(r["energy"], e) < 1e-9 and r["accepted_iterations"] == acc and r["stop_reason"] == stop
    np.testing.assert_allclose(out["warm_start_params"], g["warm_start_params"], atol=1e-6)
    assert rel(out["warm_start_energy"], g["warm_start_energy"]) < 1e-9
    assert out["global_result"]["accepted_iterations"] == g["global_accepted"]
    assert rel(out["global_result"]["energy"], g["global_energy"]) < 1e-9
    assert rel(out["best_energy"], g["best_energy"]) < 1e-9
    np.testing.assert_allclose(out["best_params"], g["best_params"], atol=1e-6)
    eng.close()


def test_sample_counts_in_protein_decoder_order(vq):
    """A 7-qubit computational state with qubit 0 flipped samples as '1000000'
    (qubit 0 leftmost, the plugin's key order); the decoder's order puts qubit 0
    rightmost (the reference's readout test, test/tests/test_readout.py:14-15)."""
    from vqemps import ingest, shim
    kernel = shim.make_kernel()
    q = kernel.qalloc(7)
    kernel.x(q[0])
    counts = shim.sample(kernel, shots_count=1000)
    assert dict(counts) == {"1000000": 1000}
    assert ingest.protein_probabilities(counts) == {"0000001": 1.0}
    kernel2, theta = shim.make_kernel(float)
    r = kernel2.qalloc(7)
    kernel2.x(r[2])
    kernel2.ry(theta, r[6])
    counts2 = shim.sample(kernel2, 2.0 * np.arccos(np.sqrt(0.75)), shots_count=4000)
    probs = ingest.protein_probabilities(counts2)
    assert set(probs) == {"0000100", "1000100"} and abs(probs["0000100"] - 0.75) < 0.04
