"""The oracle pinned against the reference: golden vectors of its own ReverseMPS
(tests/golden/make_golden.py) and the known answers of its validation scripts."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import mps_oracle as O
from oracle import workloads as W

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reverse_mps_golden.json").read_text())


def _spec(case):
    s = case["spec"]
    return dict(n=s["n"], ops=[tuple(o) for o in s["ops"]], initial=s["initial"], count=s["count"])


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_oracle_energy_matches_reference_reverse_mps(case):
    spec = _spec(case)
    e = O.reverse_energy(spec, case["words"], np.array(case["coeffs"]), np.array(case["x"]))
    assert abs(e - case["energy"]) <= 1e-10 * max(1.0, abs(case["energy"]))


@pytest.mark.parametrize("case", [c for c in GOLDEN if c["gradient"] is not None and c["spec"]["n"] <= 12],
                         ids=lambda c: c["name"])
def test_oracle_gradient_matches_reference_reverse_mps(case):
    spec = _spec(case)
    e, g = O.reverse_value_gradient(spec, case["words"], np.array(case["coeffs"]), np.array(case["x"]))
    ref = np.array(case["gradient"])
    assert abs(e - case["energy"]) <= 1e-10 * max(1.0, abs(case["energy"]))
    np.testing.assert_allclose(g, ref, rtol=1e-9, atol=1e-9 * max(1.0, np.abs(ref).max()))


@pytest.mark.parametrize("case", [c for c in GOLDEN if c["spec"]["n"] <= 12], ids=lambda c: c["name"])
def test_svd_evolution_state_equals_exact_state(case):
    """The plugin's SVD path (zero cutoff, exact cap) prepares the same state."""
    spec = _spec(case)
    x = np.array(case["x"])
    ss = O.svd_evolve(spec, x, 16)
    psi = O.statevector(ss)
    dense = O.dense_statevector(spec, x)
    np.testing.assert_allclose(psi, dense, atol=1e-12)
    e = float(np.dot(O.expect_words(ss, case["words"]).real, case["coeffs"]))
    assert abs(e - case["energy"]) <= 1e-10 * max(1.0, abs(case["energy"]))


def two_qubit_known_answer():
    """setup_local_cudaq.sh:3019-3061: ry(t) q0; x q1; cx q0 q1 and a 7-term H."""
    ops = [("ry", 0, 0), ("x", 1), ("cx", 0, 1)]
    paulis = ["II", "ZI", "IZ", "XX", "YY", "ZZ", "IX"]      # qubit order
    coeffs = [0.11] + [0.11 + 0.03 * k for k in range(1, 7)]
    return ops, paulis, coeffs


def test_two_qubit_closed_form():
    ops, words, coeffs = two_qubit_known_answer()
    spec = dict(n=2, ops=ops, initial=None, count=1)
    t = 0.37
    expected = -0.15 + 0.43 * math.sin(t) - 0.03 * math.cos(t)
    e = float(np.dot(O.dense_expectations(O.dense_statevector(spec, [t]), words).real, coeffs))
    assert abs(e - expected) < 1e-10
    ss = O.svd_evolve(spec, [t], 2)
    assert abs(float(np.dot(O.expect_words(ss, words).real, coeffs)) - expected) < 1e-10


@pytest.mark.parametrize("width", [2, 5, 3, 2])
def test_changing_register_widths(width):
    """setup_local_cudaq.sh:3088-3097: Z0 + 0.25 Z_{w-1} after ry(t) on q0 is cos t + 0.25."""
    t = 0.37
    spec = dict(n=width, ops=[("ry", 0, 0)], initial=None, count=1)
    words = ["Z" + "I" * (width - 1), "I" * (width - 1) + "Z"]
    ss = O.svd_evolve(spec, [t], 16)
    e = float(np.dot(O.expect_words(ss, words).real, [1.0, 0.25]))
    assert abs(e - (math.cos(t) + 0.25)) < 1e-10


def test_chunk_size_invariance():
    """test_reverse_mps.py:76-78: chunking changes neither energy nor gradient."""
    case = next(c for c in GOLDEN if c["name"] == "unit_test_circuit")
    spec = _spec(case)
    e1 = O.reverse_energy(spec, case["words"], np.array(case["coeffs"]), np.array(case["x"]), chunk=1)
    e2 = O.reverse_energy(spec, case["words"], np.array(case["coeffs"]), np.array(case["x"]), chunk=128)
    assert abs(e1 - e2) < 1e-12


def test_configure_full_bond_values():
    """validate_mps.py:25-30."""
    assert O.configure_full_bond(6) == 8
    assert O.configure_full_bond(62) == 2 ** 31 - 1
    assert O.configure_full_bond(97) == 2 ** 31 - 1
    assert O.configure_full_bond(97, [{"entanglement": "linear", "reps": 4}]) == 16
    assert O.configure_full_bond(97, [{"entanglement": "reverse_linear", "reps": 4}]) == 16
    assert O.configure_full_bond(97, [{"entanglement": "pairwise", "reps": 4}]) == 4


def test_allocation_bound_97_qubits():
    """test_graph_resources.py:10-16: a 97-qubit nearest-neighbour chain stays at 16."""
    for reverse in (False, True):
        edges = [(i, i + 1) for i in range(96)]
        if reverse:
            edges.reverse()
        bonds = O.allocation_bonds(97, edges * 4, 16)
        assert max(bonds) == 16


def test_rank_guard_fires_when_cap_is_too_small():
    spec, words, coeffs, x = W.plain_12q(3)
    with pytest.raises(O.InsufficientBond):
        O.svd_evolve(spec, x, 4)


def test_cap_16_and_32_agree():
    """validate_mps_97.py:109-114: an exact cap and a larger one give the same energy."""
    spec, words, coeffs, x = W.plain_12q(5)
    e16 = float(np.dot(O.expect_words(O.svd_evolve(spec, x, 16), words).real, coeffs))
    e32 = float(np.dot(O.expect_words(O.svd_evolve(spec, x, 32), words).real, coeffs))
    assert abs(e16 - e32) <= 1e-9 * max(1.0, abs(e16))


def test_philox_known_answers():
    """Random123 known-answer vectors of Philox4x32-10."""
    assert O.philox4x32([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert O.philox4x32([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert O.philox4x32([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_fnv_word_seed_and_shard_seed():
    # FNV-1a of the empty string is the offset basis (xor the evaluation seed)
    assert O.seed_for_word(0, "") == 2166136261
    assert O.seed_for_word(5, "") == 2166136261 ^ 5
    # hand-evaluated FNV-1a("Z") with seed 0
    assert O.seed_for_word(0, "Z") == ((2166136261 ^ ord("Z")) * 16777619) & 0xFFFFFFFF
    v = O.seed_for_shot_shard(1234567, 0)
    assert 0 <= v < 2 ** 32 and v != O.seed_for_shot_shard(1234568, 0)


def test_perfect_sampling_matches_exact_distribution():
    """Perfect sampling reproduces |psi|^2 (chi-square at 5 qubits, 4000 shots)."""
    from scipy.stats import chi2
    spec = O.hardware_efficient_spec(5, 2, ("ry",), "linear")
    x = np.random.default_rng(11).uniform(-np.pi, np.pi, spec["count"])
    sites = O.svd_evolve(spec, x, 4)
    probs = O.exact_probabilities(sites)
    for rng in ("splitmix", "philox"):
        bits = O.sample_bits(sites, 4000, 99, rng)
        idx = bits.astype(np.int64) @ (1 << np.arange(4, -1, -1))
        obs = np.bincount(idx, minlength=32)
        keep = probs * 4000 > 5
        exp = probs[keep] * 4000
        stat = np.sum((obs[keep] - exp) ** 2 / exp) + (obs[~keep].sum() - probs[~keep].sum() * 4000) ** 2 / max(probs[~keep].sum() * 4000, 1e-9)
        assert stat < chi2.ppf(0.999, keep.sum())


def test_reverse_chain_keeps_state():
    spec, words, coeffs, x = W.plain_12q(1)
    ss = O.svd_evolve(spec, x, 16)
    rev = O.reverse_chain(ss)
    psi = O.statevector(ss).reshape([2] * 12)
    psi_rev = O.statevector(rev).reshape([2] * 12)
    np.testing.assert_allclose(np.transpose(psi_rev, list(range(11, -1, -1))), psi, atol=1e-13)


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_cpu_baseline_matches_reference(case):
    """The timed C restatement (oracle/cpu_energy.c) gives the reference's energies."""
    from oracle import cpu_baseline
    spec = _spec(case)
    e = cpu_baseline.energy(spec, case["words"], np.array(case["coeffs"]), np.array(case["x"]), threads=4)
    assert abs(e - case["energy"]) <= 1e-10 * max(1.0, abs(case["energy"]))


def test_z_sample_sums_on_unsigned_bits():
    bits = np.array([[1, 0, 1], [0, 0, 1]], dtype=np.uint8)
    assert list(O.z_sample_sums(bits, ["ZZI", "IIZ", "III"])) == [0, -2, 2]


def test_product_workloads_equal_the_oracle_workloads():
    """bench.py and the benchmarks draw their inputs from vqemps.workloads; the
    tests from oracle.workloads: the two generators give the same instances."""
    from oracle import workloads as OW
    from vqemps import workloads as PW
    a, b = OW.batched_40q(seed=3, batch=8), PW.batched_40q(seed=3, batch=8)
    assert a[0]["ops"] == [tuple(o) for o in b[0]["ops"]] and a[1] == b[1]
    assert np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])
    pa, pb = OW.uneven_partitions(seed=1, partitions=3), PW.uneven_partitions(seed=1, partitions=3)
    for x, y in zip(pa, pb):
        assert x[0]["ops"] == y[0]["ops"] and x[1] == y[1] and np.array_equal(x[2], y[2])
    g1, g2 = OW.gradient_64q(seed=2, batch=2, terms=50), PW.gradient_64q(seed=2, batch=2, terms=50)
    assert g1[1] == g2[1] and np.array_equal(g1[3], g2[3]) and g1[0]["ops"] == g2[0]["ops"]
    p1, p2 = OW.plain_12q(1), PW.plain_12q(1)
    assert p1[1] == p2[1] and np.array_equal(p1[3], p2[3])
