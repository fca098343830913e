"""Benchmark-size parity against the reference's own ReverseMPS.

* The benchmark batch (40 qubits, reverse_linear, 5,000 terms, B = 256 SPSA
  probes, ``vqemps.workloads.batched_40q(seed=0)``): four of the timed
  parameter sets, evaluated inside the full B = 256 call, against the
  reference's energies (1e-9 relative).
* The gradient workload (64 qubits, linear, 320 angles, 20,000 terms of weight
  <= 6, B = 32, environments checkpointed every 8 levels, split plan chosen by
  the planner): energies (1e-9 relative) and full gradients (1e-8 of the largest
  component) of two parameter sets against the reference's ``value_gradient``,
  and 16 gradient components against FP64 central differences (h = 1e-4) of the
  engine's energy (1e-5 relative).

The golden values come from tests/golden/make_golden.py --large, which runs the
reference's ReverseMPS on the CPU; the workloads are regenerated here and
checked against the recorded digests first.
"""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
LARGE = json.loads((Path(__file__).parent / "golden" / "large_workloads_golden.json").read_text())


@pytest.fixture(scope="module")
def vq(cuda_device):
    import vqemps
    return vqemps


@pytest.mark.parametrize("variant", [None, "dmma3_pf", "dmma_pf"])
def test_bench_batch_matches_reference_energies(vq, variant):
    from vqemps import workloads as VW
    spec, words, coeffs, thetas = VW.batched_40q(seed=0, batch=256)
    g = LARGE["batched_40q"]
    assert VW.workload_digest(words, coeffs) == g["digest"]
    eng = vq.Engine(0, 16)
    eng.set_spec(spec)
    if variant is not None:
        eng.set_level_variant(variant)
    ham = eng.set_hamiltonian(words, coeffs)
    e = eng.energy(ham, torch.tensor(thetas, device=eng.device)).cpu().numpy()
    assert e.shape == (256,) and np.isfinite(e).all()
    for i, ref in zip(g["indices"], g["energies"]):
        assert abs(e[i] - ref) <= 1e-9 * max(1.0, abs(ref)), (i, e[i], ref)
    eng.close()


@pytest.fixture(scope="module")
def grad64(vq):
    from vqemps import workloads as VW
    spec, words, coeffs, thetas = VW.gradient_64q(seed=0, batch=32)
    g = LARGE["gradient_64q"]
    assert VW.workload_digest(words, coeffs) == g["digest"]
    return spec, words, coeffs, thetas, g


@pytest.mark.parametrize("variant", ["dmma3", "dmma"])
def test_gradient_64q_matches_reference_golden(vq, grad64, variant):
    spec, words, coeffs, thetas, g = grad64
    eng = vq.Engine(0, 16)
    eng.set_grad_checkpoint(8)
    eng.set_grad_variant(variant)
    eng.set_spec(spec)
    ham = eng.set_hamiltonian(words, coeffs)
    assert eng.plan_stats(ham)["cut"] > 0       # the planner picks the split evaluation here
    e, grad = eng.energy_grad(ham, torch.tensor(thetas, device=eng.device))
    e, grad = e.cpu().numpy(), grad.cpu().numpy()
    assert e.shape == (32,) and grad.shape == (32, 320)
    e_only = eng.energy(ham, torch.tensor(thetas, device=eng.device)).cpu().numpy()
    np.testing.assert_allclose(e, e_only, rtol=1e-11)
    for k, i in enumerate(g["indices"]):
        ref_e, ref_g = g["energies"][k], np.array(g["gradients"][k])
        assert abs(e[i] - ref_e) <= 1e-9 * max(1.0, abs(ref_e)), (i, e[i], ref_e)
        np.testing.assert_allclose(grad[i], ref_g, rtol=0, atol=1e-8 * max(1.0, np.abs(ref_g).max()))
    eng.close()


def test_gradient_64q_central_differences(vq, grad64):
    spec, words, coeffs, thetas, g = grad64
    eng = vq.Engine(0, 16)
    eng.set_grad_checkpoint(8)
    eng.set_spec(spec)
    ham = eng.set_hamiltonian(words, coeffs)
    theta = thetas[5]
    _, grad = eng.energy_grad(ham, torch.tensor(theta[None], device=eng.device))
    grad = grad[0].cpu().numpy()
    h = 1e-4
    idx = np.linspace(0, spec["count"] - 1, 16).astype(int)
    pts = np.repeat(theta[None], 32, 0)
    pts[np.arange(16), idx] += h
    pts[16 + np.arange(16), idx] -= h
    e = eng.energy(ham, torch.tensor(pts, device=eng.device)).cpu().numpy()
    fd = (e[:16] - e[16:]) / (2 * h)
    np.testing.assert_allclose(grad[idx], fd, rtol=1e-5, atol=1e-5 * np.abs(grad).max())
    eng.close()
