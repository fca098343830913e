"""GPU adjoint gradient parity: the reference's ReverseMPS golden gradients,
the oracle's adjoint, and FP64 central differences (h = 1e-4) of the engine's
own energy. Tolerance: 1e-8 relative to the largest component (golden/oracle),
1e-5 relative for central differences."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import mps_oracle as O
from oracle import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "reverse_mps_golden.json").read_text())


@pytest.fixture(scope="module")
def vq(cuda_device):
    import vqemps
    return vqemps


def _spec(case):
    s = case["spec"]
    return dict(n=s["n"], ops=[tuple(o) for o in s["ops"]], initial=s["initial"], count=s["count"])


@pytest.mark.parametrize("case", [c for c in GOLDEN if c["gradient"] is not None], ids=lambda c: c["name"])
@pytest.mark.parametrize("order", ["msb", "qubit"])
@pytest.mark.parametrize("every", [1, 3, 8])
@pytest.mark.parametrize("variant", ["dmma3", "dmma", "simt"])
def test_gradient_matches_reference_golden(vq, case, order, every, variant):
    spec = _spec(case)
    eng = vq.Engine(0, 16)
    eng.set_grad_checkpoint(every)
    eng.set_grad_variant(variant)
    eng.set_spec(spec, site_order=order)
    ham = eng.set_hamiltonian(case["words"], case["coeffs"])
    e, g = eng.energy_grad(ham, np.array(case["x"]))
    ref = np.array(case["gradient"])
    assert abs(float(e[0]) - case["energy"]) <= 1e-9 * max(1.0, abs(case["energy"]))
    np.testing.assert_allclose(g[0].cpu().numpy(), ref, rtol=0, atol=1e-8 * max(1.0, np.abs(ref).max()))


def test_gradient_batch_and_central_differences(vq):
    spec, words, coeffs, theta = W.plain_12q(2)
    eng = vq.Engine(0, 16)
    eng.set_spec(spec)
    ham = eng.set_hamiltonian(words, coeffs)
    th = np.stack([theta, theta * 0.5])
    e, g = eng.energy_grad(ham, th)
    e2 = eng.energy(ham, th).cpu().numpy()
    np.testing.assert_allclose(e.cpu().numpy(), e2, rtol=1e-10)
    h = 1e-4
    idx = np.arange(0, spec["count"], 7)
    plus = np.repeat(theta[None], len(idx), 0)
    minus = plus.copy()
    plus[np.arange(len(idx)), idx] += h
    minus[np.arange(len(idx)), idx] -= h
    fd = (eng.energy(ham, plus).cpu().numpy() - eng.energy(ham, minus).cpu().numpy()) / (2 * h)
    gg = g[0].cpu().numpy()[idx]
    np.testing.assert_allclose(gg, fd, rtol=1e-5, atol=1e-5 * np.abs(gg).max())
    _, gref = O.reverse_value_gradient(spec, words, coeffs, theta)
    np.testing.assert_allclose(g[0].cpu().numpy(), gref, atol=1e-8 * np.abs(gref).max())


def test_gradient_with_identity_and_offdiagonal_terms(vq):
    spec = dict(n=3, initial="+", count=4,
                ops=[("ry", 0, 0), ("rz", 1, 1), ("cx", 1, 0), ("rx", 2, 2), ("cx", 1, 2), ("ry", 1, 3)])
    words = ["YXI", "ZZI", "III", "XXZ", "IIY"]
    coeffs = np.array([.3, -.7, .4, .2, 1.5])
    x = np.array([.2, -.4, .8, .1])
    eng = vq.Engine(0, 16)
    eng.set_spec(spec)
    ham = eng.set_hamiltonian(words, coeffs)
    e, g = eng.energy_grad(ham, x)
    eref, gref = O.reverse_value_gradient(spec, words, coeffs, x)
    assert abs(float(e[0]) - eref) < 1e-12
    np.testing.assert_allclose(g[0].cpu().numpy(), gref, atol=1e-11)


def test_checkpointing_is_bitwise_neutral(vq):
    """Recomputed environments are the same numbers: every interval gives the same bits."""
    spec, words, coeffs, theta = W.plain_12q(4)
    out = []
    for every in (1, 2, 5, 8, 40):
        eng = vq.Engine(0, 16)
        eng.set_grad_checkpoint(every)
        eng.set_spec(spec)
        ham = eng.set_hamiltonian(words, coeffs)
        e, g = eng.energy_grad(ham, np.stack([theta, -theta]))
        out.append((e.cpu().numpy(), g.cpu().numpy()))
    for e, g in out[1:]:
        assert np.array_equal(e, out[0][0]) and np.array_equal(g, out[0][1])


def test_dmma_and_simt_gradient_kernels_agree(vq):
    """The FP64 tensor-core gradient levels and the SIMT ones compute the same
    products in another summation order: equal to rounding at 40 qubits."""
    import torch
    spec, words, coeffs, thetas = W.batched_40q(seed=4, batch=4, terms=2000)
    out = {}
    for variant in ("dmma3", "dmma", "simt"):
        eng = vq.Engine(0, 16)
        eng.set_spec(spec)
        eng.set_grad_variant(variant)
        ham = eng.set_hamiltonian(words, coeffs)
        e, g = eng.energy_grad(ham, torch.tensor(thetas, device=eng.device))
        out[variant] = (e.cpu().numpy(), g.cpu().numpy())
    e2, g2 = out["simt"]
    for variant in ("dmma3", "dmma"):
        e1, g1 = out[variant]
        assert np.allclose(e1, e2, rtol=1e-12, atol=1e-9)
        assert np.abs(g1 - g2).max() <= 1e-10 * max(1.0, np.abs(g2).max())
