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
