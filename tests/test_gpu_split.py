"""GPU: split evaluation (prefix trie up to a cut site, suffix trie from it, one
dot product per prefix/suffix pair) against the prefix trie alone and the
oracle. Same values to rounding: 1e-12 relative between the two plans, the usual
1e-9 against the oracle."""
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


def _energies(vq, spec, words, coeffs, thetas, mode, variant=None, order="msb"):
    eng = vq.Engine(0, 16)
    eng.set_spec(spec, site_order=order)
    eng.set_split_mode(mode)
    eng.set_level_variant(variant)
    ham = eng.set_hamiltonian(words, coeffs)
    e, pt = eng.energy(ham, thetas, per_term=True)
    return e.cpu().numpy(), pt.cpu().numpy(), eng.plan_stats(ham)


@pytest.mark.parametrize("order", ["msb", "qubit"])
@pytest.mark.parametrize("case", [c for c in GOLDEN if c["spec"]["n"] >= 3], ids=lambda c: c["name"])
def test_forced_split_matches_golden_and_prefix_plan(vq, case, order):
    spec = _spec(case)
    x = np.array(case["x"])
    e1, pt1, st1 = _energies(vq, spec, case["words"], case["coeffs"], x, "on", order=order)
    e0, pt0, st0 = _energies(vq, spec, case["words"], case["coeffs"], x, "off", order=order)
    assert st1["cut"] >= 1 and st0["cut"] == -1
    assert abs(e1[0] - case["energy"]) <= 1e-9 * max(1.0, abs(case["energy"]))
    assert abs(e1[0] - e0[0]) <= 1e-12 * max(1.0, abs(e0[0]))
    np.testing.assert_allclose(pt1, pt0, rtol=0, atol=1e-12)


@pytest.mark.parametrize("variant", [None, "simt", "dmma_pf", "dmma3_pf"])
def test_auto_split_at_40_qubits(vq, variant):
    """The 40-qubit, 5,000-term plan splits by itself and needs about half the
    node-sites; every level-kernel variant gives the same energies and per-term
    values as the prefix plan."""
    spec, words, coeffs, thetas = W.batched_40q(2, batch=8)
    words = list(words) + ["I" * 40]                       # an identity word as well
    coeffs = np.append(coeffs, 3.5)
    e1, pt1, st1 = _energies(vq, spec, words, coeffs, thetas, "auto", variant)
    e0, pt0, st0 = _energies(vq, spec, words, coeffs, thetas, "off", variant)
    assert 1 <= st1["cut"] < 39 and st1["node_sites"] < 0.6 * st1["prefix_node_sites"]
    assert st1["pairs"] > 0
    np.testing.assert_allclose(e1, e0, rtol=1e-12)
    np.testing.assert_allclose(pt1, pt0, rtol=0, atol=1e-11)
    ref = float(np.dot(O.expect_words(O.svd_evolve(spec, thetas[3], 16), words).real, coeffs))
    assert abs(e1[3] - ref) <= 1e-9 * max(1.0, abs(ref))


def test_per_term_cuts_at_40_qubits(vq):
    """The benchmark's Hamiltonian: closing each word at its own cut needs fewer
    node-sites than the single cut at site 20 (18,913); a batch of 32 states uses
    it, and its energies and per-term values equal the prefix plan's for the real
    and the complex level kernels."""
    spec, words, coeffs, thetas = W.batched_40q(0, batch=32)
    for variant in ("real_pf", "dmma3_pf"):
        e1, pt1, st1 = _energies(vq, spec, words, coeffs, thetas, "auto", variant)
        e0, pt0, st0 = _energies(vq, spec, words, coeffs, thetas, "off", variant)
        assert st1["cut"] == 20 and st1["node_sites"] <= 16000 and st1["pairs"] > 3000
        np.testing.assert_allclose(e1, e0, rtol=1e-12)
        np.testing.assert_allclose(pt1, pt0, rtol=0, atol=1e-11)
        # a small batch evaluates the same states with the single cut
        e4, pt4, _ = _energies(vq, spec, words, coeffs, thetas[:4], "auto", variant)
        np.testing.assert_allclose(e4, e1[:4], rtol=1e-12)
        np.testing.assert_allclose(pt4, pt1[:4], rtol=0, atol=1e-11)


def test_split_with_sampling_and_widths(vq):
    """Shot estimates use the split plan's analytic X/Y values; tiny widths and
    words ending on either side of the cut."""
    rng = np.random.default_rng(5)
    from oracle.workloads import random_hamiltonian
    for n in (3, 4, 9):
        spec = O.hardware_efficient_spec(n, 3, ("ry", "rz"), "linear")
        words, coeffs = random_hamiltonian(rng, n, 40, 3, z_fraction=0.6)
        words[0] = "I" * n
        x = rng.uniform(-np.pi, np.pi, spec["count"])
        out = {}
        for mode in ("on", "off"):
            eng = vq.Engine(0, 16)
            eng.set_spec(spec)
            eng.set_split_mode(mode)
            ham = eng.set_hamiltonian(words, coeffs)
            e, pt = eng.sampled_energy(ham, x, 500, 11, "philox", "shared", per_term=True)
            out[mode] = (e.cpu().numpy(), pt.cpu().numpy(), eng.plan_stats(ham)["cut"])
        assert out["on"][2] >= 1
        np.testing.assert_allclose(out["on"][1], out["off"][1], rtol=0, atol=1e-12)
        np.testing.assert_allclose(out["on"][0], out["off"][0], rtol=1e-12, atol=1e-12)


def _grad(vq, spec, words, coeffs, thetas, mode, variant="dmma3", every=8, order="msb"):
    eng = vq.Engine(0, 16)
    eng.set_spec(spec, site_order=order)
    eng.set_split_mode(mode)
    eng.set_grad_variant(variant)
    eng.set_grad_checkpoint(every)
    ham = eng.set_hamiltonian(words, coeffs)
    e, g = eng.energy_grad(ham, thetas)
    return e.cpu().numpy(), g.cpu().numpy(), eng.plan_stats(ham)


@pytest.mark.parametrize("variant", ["dmma3", "dmma"])
@pytest.mark.parametrize("every", [1, 3])
@pytest.mark.parametrize("order", ["msb", "qubit"])
@pytest.mark.parametrize("case", [c for c in GOLDEN if c["spec"]["n"] >= 3 and c["gradient"] is not None],
                         ids=lambda c: c["name"])
def test_split_gradient_matches_golden(vq, case, order, every, variant):
    """Adjoint gradient through the split evaluation (pair cotangents, suffix
    levels on transposed sites, cotangents of the suffix roots' R_{l+1}) against
    the reference's ReverseMPS gradients: 1e-8 of the largest component."""
    spec = _spec(case)
    e, g, st = _grad(vq, spec, case["words"], case["coeffs"], np.array(case["x"]), "on", variant, every, order)
    assert st["cut"] >= 1
    ref = np.array(case["gradient"])
    assert abs(float(e[0]) - case["energy"]) <= 1e-9 * max(1.0, abs(case["energy"]))
    np.testing.assert_allclose(g[0], ref, rtol=0, atol=1e-8 * max(1.0, np.abs(ref).max()))


def test_split_gradient_at_40_qubits(vq):
    """40 qubits, 2,000 terms plus an identity word, four parameter sets: the
    split gradient equals the prefix plan's to rounding and matches FP64
    central differences of the engine's energy."""
    spec, words, coeffs, thetas = W.batched_40q(seed=6, batch=4, terms=2000)
    words = list(words) + ["I" * 40]
    coeffs = np.append(coeffs, -1.25)
    e1, g1, st1 = _grad(vq, spec, words, coeffs, thetas, "on")
    e0, g0, st0 = _grad(vq, spec, words, coeffs, thetas, "off")
    assert st1["cut"] >= 1 and st0["cut"] == -1
    np.testing.assert_allclose(e1, e0, rtol=1e-12)
    assert np.abs(g1 - g0).max() <= 1e-10 * max(1.0, np.abs(g0).max())
    eng = vq.Engine(0, 16)
    eng.set_spec(spec)
    ham = eng.set_hamiltonian(words, coeffs)
    h = 1e-4
    idx = np.arange(0, spec["count"], 23)
    plus = np.repeat(thetas[1][None], len(idx), 0)
    minus = plus.copy()
    plus[np.arange(len(idx)), idx] += h
    minus[np.arange(len(idx)), idx] -= h
    fd = (eng.energy(ham, plus).cpu().numpy() - eng.energy(ham, minus).cpu().numpy()) / (2 * h)
    np.testing.assert_allclose(g1[1][idx], fd, rtol=1e-5, atol=1e-5 * np.abs(g1[1]).max())


def test_split_gradient_with_words_on_both_sides_of_the_cut(vq):
    """Small widths, forced split, words ending before, at and after the cut,
    identity and off-diagonal words: split gradient equals the prefix plan's."""
    rng = np.random.default_rng(11)
    from oracle.workloads import random_hamiltonian
    for n in (3, 4, 7, 12):
        spec = O.hardware_efficient_spec(n, 3, ("ry", "rz"), "reverse_linear")
        words, coeffs = random_hamiltonian(rng, n, 60, 4, z_fraction=0.5)
        words[0] = "I" * n
        x = rng.uniform(-np.pi, np.pi, (3, spec["count"]))
        e1, g1, st1 = _grad(vq, spec, words, coeffs, x, "on", every=2)
        e0, g0, _ = _grad(vq, spec, words, coeffs, x, "off", every=2)
        assert st1["cut"] >= 1
        np.testing.assert_allclose(e1, e0, rtol=1e-12, atol=1e-12)
        assert np.abs(g1 - g0).max() <= 1e-11 * max(1.0, np.abs(g0).max())
