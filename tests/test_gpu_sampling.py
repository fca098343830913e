"""GPU sampling parity: reference-exact SplitMix shots, Philox distribution
(chi-square against the exact probabilities) and shot-estimated energies."""
import numpy as np
import pytest
import torch
from scipy.stats import chi2

from oracle import mps_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vq(cuda_device):
    import vqemps
    return vqemps


def _prep(vq, n=6, reps=3, seed=4, order="msb"):
    spec = O.hardware_efficient_spec(n, reps, ("ry", "rz"), "linear")
    x = np.random.default_rng(seed).uniform(-np.pi, np.pi, spec["count"])
    eng = vq.Engine(0, 16)
    eng.set_spec(spec, site_order=order)
    return spec, x, eng


def test_splitmix_shots_are_the_plugins_shots(vq):
    """With the plugin's msb sites and SplitMix draws every shot equals the
    oracle's restatement of sampleBitsFromPreparedRight bit for bit."""
    spec, x, eng = _prep(vq)
    n = spec["n"]
    ev_seed = 1234567
    bits = eng.sample(x, 300, ev_seed, "splitmix")
    got = vq.unpack_bits(bits, n)[0]
    sites = O.reverse_chain(O.svd_evolve(spec, x, 16))        # plugin site order
    draw_seed = O.seed_for_shot_shard(ev_seed, 0)
    ref_site = O.sample_bits(sites, 300, draw_seed, "splitmix")
    ref_qubit = ref_site[:, ::-1]                              # site s = qubit n-1-s
    assert np.array_equal(got, ref_qubit)


def test_philox_matches_exact_distribution(vq):
    spec, x, eng = _prep(vq, n=5, reps=2, seed=8, order="qubit")
    shots = 8192
    bits = eng.sample(x, shots, 77, "philox")
    arr = vq.unpack_bits(bits, 5)[0]
    idx = arr.astype(np.int64) @ (1 << np.arange(4, -1, -1))
    obs = np.bincount(idx, minlength=32)
    probs = np.abs(O.dense_statevector(spec, x)) ** 2
    keep = probs * shots > 5
    exp = probs[keep] * shots
    rest_e = probs[~keep].sum() * shots
    stat = np.sum((obs[keep] - exp) ** 2 / exp) + ((obs[~keep].sum() - rest_e) ** 2 / rest_e if rest_e > 0 else 0)
    assert stat < chi2.ppf(0.999, keep.sum())


def test_philox_uniforms_match_oracle_and_draws_differ_per_state(vq):
    spec, x, eng = _prep(vq, n=6, order="qubit")
    th = np.stack([x, x])
    bits = eng.sample(th, 200, 5, "philox")
    a = vq.unpack_bits(bits, 6)
    assert not np.array_equal(a[0], a[1])        # state b draws with seed + b
    ref = O.sample_bits(O.svd_evolve(spec, x, 16), 200, 5, "philox")
    assert np.array_equal(a[0], ref)


def test_shot_energy_shared_set_equals_counts_estimate(vq):
    """Shared mode: every Z word estimated from the same bits (k_zSampleSums)."""
    spec, x, eng = _prep(vq, n=7, reps=3, seed=2)
    rng = np.random.default_rng(0)
    from oracle.workloads import random_hamiltonian
    words, coeffs = random_hamiltonian(rng, 7, 60, 4, z_fraction=0.8)
    words[0] = "I" * 7
    ham = eng.set_hamiltonian(words, coeffs)
    shots, seed = 2048, 99
    e, pt = eng.sampled_energy(ham, x, shots, seed, "splitmix", "shared", per_term=True)
    bits = vq.unpack_bits(eng.sample(x, shots, seed, "splitmix"), 7)[0]
    sums = O.z_sample_sums(bits, words)
    exact = O.expect_words(O.svd_evolve(spec, x, 16), words).real
    vals = np.array([exact[t] if any(c in "XY" for c in w) else sums[t] / shots for t, w in enumerate(words)])
    np.testing.assert_allclose(pt[0].cpu().numpy(), vals, atol=1e-11)
    assert abs(float(e[0]) - float(np.dot(vals, coeffs))) < 1e-9 * max(1, np.abs(coeffs).sum())
    # statistically close to the analytic energy
    sigma = np.sqrt(np.sum(coeffs ** 2 * (1 - np.minimum(exact ** 2, 1)))) / np.sqrt(shots)
    assert abs(float(e[0]) - float(np.dot(exact, coeffs))) < 6 * sigma + 1e-9


def test_shot_energy_plugin_mode_independent_streams(vq):
    """Plugin mode with X/Y words: one stream per Z word with its FNV seed."""
    spec, x, eng = _prep(vq, n=6, reps=2, seed=9)
    words = ["ZIIIII", "IZZIII", "XIIIII", "IIIIZZ", "IIIIII", "YZIIIX"]
    coeffs = np.array([0.7, -0.3, 0.5, 1.1, 0.2, -0.4])
    ham = eng.set_hamiltonian(words, coeffs)
    shots, ev = 1000, 42
    e, pt = eng.sampled_energy(ham, x, shots, ev, "splitmix", "plugin", per_term=True)
    sites = O.reverse_chain(O.svd_evolve(spec, x, 16))
    exact = O.expect_words(O.svd_evolve(spec, x, 16), words).real
    for t, w in enumerate(words):
        got = float(pt[0, t])
        if "X" in w or "Y" in w:
            assert abs(got - exact[t]) < 1e-11
        elif set(w) == {"I"}:
            assert got == 1.0
        else:
            site_word = w[::-1]
            seed = O.seed_for_word(ev, site_word)
            b = O.sample_bits(sites, shots, seed, "splitmix")[:, ::-1]
            assert got == O.z_sample_sums(b, [w])[0] / shots
