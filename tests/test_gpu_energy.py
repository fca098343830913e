"""GPU parity of state preparation and analytic energies against the oracle.

Tolerances: energies within 1e-9 relative of the complex128 oracle / the
reference's ReverseMPS (FP64 throughout); statevectors within 1e-11 absolute.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import mps_oracle as O
from oracle import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "reverse_mps_golden.json").read_text())
RTOL = 1e-9


def _spec(case):
    s = case["spec"]
    return dict(n=s["n"], ops=[tuple(o) for o in s["ops"]], initial=s["initial"], count=s["count"])


@pytest.fixture(scope="module")
def vq(cuda_device):
    import vqemps
    return vqemps


def _engine(vq, spec, max_bond=16, order="msb"):
    eng = vq.Engine(0, max_bond)
    eng.set_spec(spec, site_order=order)
    return eng


@pytest.mark.parametrize("variant", ["simt", "dmma4", "dmma8", "simt_pf", "dmma_pf", "dmma3_pf"])
@pytest.mark.parametrize("order", ["msb", "qubit"])
@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_energy_matches_reference_golden(vq, case, order, variant):
    spec = _spec(case)
    eng = _engine(vq, spec, order=order)
    eng.set_level_variant(variant)
    ham = eng.set_hamiltonian(case["words"], case["coeffs"])
    e = float(eng.energy(ham, np.array(case["x"]))[0])
    assert abs(e - case["energy"]) <= RTOL * max(1.0, abs(case["energy"]))


def test_per_term_values_match_oracle(vq):
    spec, words, coeffs, theta = W.plain_12q(0)
    eng = _engine(vq, spec)
    ham = eng.set_hamiltonian(words, coeffs)
    e, pt = eng.energy(ham, theta, per_term=True)
    ref = O.expect_words(O.svd_evolve(spec, theta, 16), words).real
    np.testing.assert_allclose(pt[0].cpu().numpy(), ref, atol=1e-11)
    assert abs(float(e[0]) - float(np.dot(ref, coeffs))) <= RTOL * max(1.0, abs(float(e[0])))


@pytest.mark.parametrize("pattern", ["linear", "reverse_linear"])
@pytest.mark.parametrize("order", ["msb", "qubit"])
def test_prepared_state_equals_dense_state(vq, pattern, order):
    spec = O.hardware_efficient_spec(8, 3, ("ry", "rz"), pattern)
    x = np.random.default_rng(3).uniform(-np.pi, np.pi, spec["count"])
    eng = _engine(vq, spec, 8, order)
    ham = eng.set_hamiltonian(["Z" + "I" * 7], [1.0])
    eng.energy(ham, x)
    dims = eng.bond_dims()
    raw = eng.sites(0)
    sites = [raw[s, :dims[s], :, :dims[s + 1]] for s in range(8)]
    if order == "msb":
        sites = O.reverse_chain(sites)
    psi = O.statevector(sites)
    np.testing.assert_allclose(psi, O.dense_statevector(spec, x), atol=1e-11)
    # zero padding beyond the bond dims
    for s in range(8):
        blk = raw[s].copy()
        blk[:dims[s], :, :dims[s + 1]] = 0
        assert np.abs(blk).max() == 0.0


def test_bond_dims_equal_allocation_bound(vq):
    spec = O.hardware_efficient_spec(40, 4, ("ry",), "reverse_linear")
    eng = _engine(vq, spec)
    edges = [(op[1], op[2]) for op in spec["ops"] if op[0] == "cx"]
    assert eng.bond_dims() == O.allocation_bonds(40, edges, 16)


def test_rank_guard_reports_insufficient_bond(vq):
    spec, words, coeffs, theta = W.plain_12q(3)
    eng = _engine(vq, spec, max_bond=4)
    ham = eng.set_hamiltonian(words, coeffs)
    with pytest.raises(vq.EngineError, match="insufficient"):
        eng.energy(ham, theta)


def test_invalid_inputs_raise(vq):
    spec, words, coeffs, theta = W.plain_12q(0)
    eng = _engine(vq, spec)
    with pytest.raises(vq.EngineError, match="Invalid analytic Pauli"):
        eng.set_hamiltonian(["Q" + "I" * 11], [1.0])
    with pytest.raises(vq.EngineError):
        eng.set_hamiltonian(["ZI"], [1.0])
    with pytest.raises(vq.EngineError, match=">= 2 qubits"):
        eng.set_circuit(1, [("ry", 0, 0)])


def test_two_qubit_closed_form_and_widths(vq):
    t = 0.37
    eng = vq.Engine(0, 2)
    eng.set_circuit(2, [("ry", 0, 0), ("x", 1), ("cx", 0, 1)])
    ham = eng.set_hamiltonian(["II", "ZI", "IZ", "XX", "YY", "ZZ", "IX"],
                              [0.11] + [0.11 + 0.03 * k for k in range(1, 7)])
    e = float(eng.energy(ham, [t])[0])
    assert abs(e - (-0.15 + 0.43 * math.sin(t) - 0.03 * math.cos(t))) < 1e-10
    for width in (2, 5, 3, 2):
        eng = vq.Engine(0, 16)
        eng.set_circuit(width, [("ry", 0, 0)])
        ham = eng.set_hamiltonian(["Z" + "I" * (width - 1), "I" * (width - 1) + "Z"], [1.0, 0.25])
        assert abs(float(eng.energy(ham, [t])[0]) - (math.cos(t) + 0.25)) < 1e-10


@pytest.mark.parametrize("variant", ["simt", "dmma4", "dmma3_pf"])
def test_batch_equals_single_calls_bitwise(vq, variant):
    spec, words, coeffs, theta = W.plain_12q(0)
    eng = _engine(vq, spec)
    eng.set_level_variant(variant)
    ham = eng.set_hamiltonian(words, coeffs)
    th = np.stack([theta + 0.05 * k for k in range(7)])
    batch = eng.energy(ham, th).cpu().numpy()
    single = np.array([float(eng.energy(ham, t)[0]) for t in th])
    assert np.array_equal(batch, single)


def test_gates_constant_and_custom_matrices(vq):
    """Constant gates, U1/U2 matrices, non-adjacent CX (SWAP routing) vs dense."""
    rng = np.random.default_rng(5)
    q, _ = np.linalg.qr(rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)))
    q4, _ = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))
    ops = [("h", 0), ("ry", 1, 0), ("rx", 2, 1), ("u1", 3, q), ("cx", 0, 2), ("s", 1), ("sdg", 2),
           ("cx", 3, 1), ("u2", 1, 2, q4), ("rz", 0, 2), ("y", 3), ("z", 0), ("swap", 0, 3), ("x", 2)]
    x = np.array([0.3, -1.1, 0.7])
    n = 4
    # dense reference
    state = np.zeros(2 ** n, complex)
    state[0] = 1
    state = state.reshape([2] * n)

    def apply1(m, t):
        return np.moveaxis(np.tensordot(m, state, axes=([1], [t])), 0, t)

    def apply2(m4, a, b):
        g = m4.reshape(2, 2, 2, 2)
        out = np.tensordot(g, state, axes=([2, 3], [a, b]))
        return np.moveaxis(out, [0, 1], [a, b])
    mats = O.FIXED_MATRICES
    for op in ops:
        g = op[0]
        if g in ("rx", "ry", "rz"):
            state = apply1(O.rotation(g, x[op[2]]), op[1])
        elif g in mats:
            state = apply1(mats[g], op[1])
        elif g == "u1":
            state = apply1(op[2], op[1])
        elif g == "cx":
            state = apply2(O.gate4_cx(True), op[1], op[2])
        elif g == "swap":
            sw = np.zeros((4, 4))
            for i in range(2):
                for j in range(2):
                    sw[j * 2 + i, i * 2 + j] = 1
            state = apply2(sw, op[1], op[2])
        elif g == "u2":
            state = apply2(op[3], op[1], op[2])
    psi = state.reshape(-1)
    words = ["ZIII", "XYZI", "IXIY", "ZZZZ", "YIIX", "IIZX"]
    coeffs = np.array([0.5, -1.2, 0.3, 0.9, -0.4, 2.0])
    ref = float(np.dot(O.dense_expectations(psi, words).real, coeffs))
    for order in ("msb", "qubit"):
        eng = vq.Engine(0, 16)
        eng.set_circuit(n, ops, site_order=order)
        ham = eng.set_hamiltonian(words, coeffs)
        assert abs(float(eng.energy(ham, x)[0]) - ref) < 1e-11


@pytest.mark.parametrize("variant", [None, "simt", "dmma4", "dmma8", "simt_pf", "dmma_pf", "dmma3_pf"])
def test_config_40q_batch_energy_parity_sample(vq, variant):
    """40 qubits, 5,000 terms: a few probes of the SPSA batch against the oracle,
    with every trie-level kernel variant and with the autotuner's choice."""
    spec, words, coeffs, thetas = W.batched_40q(0, batch=16)
    eng = _engine(vq, spec)
    eng.set_level_variant(variant)
    ham = eng.set_hamiltonian(words, coeffs)
    e = eng.energy(ham, thetas).cpu().numpy()
    assert eng.level_variant(ham, 16) in vq.Engine.LEVEL_VARIANTS
    for b in (0, 9):
        ref = float(np.dot(O.expect_words(O.svd_evolve(spec, thetas[b], 16), words).real, coeffs))
        assert abs(e[b] - ref) <= RTOL * max(1.0, abs(ref))
    assert np.all(np.isfinite(e))


@pytest.mark.parametrize("pattern", ["linear", "reverse_linear"])
@pytest.mark.parametrize("order", ["msb", "qubit"])
def test_degenerate_angles_keep_isometric_sites(vq, pattern, order):
    """Zero and pi angles make Theta rank deficient (product or classical states):
    the left sites must stay isometries and the state must stay exact."""
    spec = O.hardware_efficient_spec(10, 4, ("ry",), pattern)
    rng = np.random.default_rng(9)
    for x in (np.zeros(spec["count"]), np.pi * rng.integers(0, 2, spec["count"]).astype(float),
              np.where(rng.random(spec["count"]) < 0.5, 0.0, rng.uniform(-np.pi, np.pi, spec["count"]))):
        eng = _engine(vq, spec, 16, order)
        ham = eng.set_hamiltonian(["Z" + "I" * 9, "IXXIIIIIII", "IIIIIYZIIX"], [1.0, 0.5, -0.25])
        eng.energy(ham, x)
        dims = eng.bond_dims()
        raw = eng.sites(0)
        sites = [raw[s, :dims[s], :, :dims[s + 1]] for s in range(10)]
        psi = O.statevector(O.reverse_chain(sites) if order == "msb" else sites)
        np.testing.assert_allclose(psi, O.dense_statevector(spec, x), atol=1e-11)
