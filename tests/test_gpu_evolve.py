"""GPU: the two-CTA gate chain (two-site gates on disjoint site pairs applied
concurrently on a schedule) gives the one-CTA program-order chain's states bit
for bit: the same gates on the same tensors, only interleaved differently."""
import numpy as np
import pytest
import torch

from oracle import mps_oracle as O
from oracle import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vq(cuda_device):
    import vqemps
    return vqemps


def _run(vq, n, ops, words, coeffs, thetas, mode, max_bond=16, order="msb"):
    eng = vq.Engine(0, max_bond)
    eng.set_evolve_mode(mode)
    eng.set_level_variant("dmma3_pf")        # the autotuner may pick differently per engine
    eng.set_circuit(n, ops, site_order=order)
    ham = eng.set_hamiltonian(words, coeffs)
    e = eng.energy(ham, torch.as_tensor(np.atleast_2d(thetas), device=eng.device)).cpu().numpy()
    return e, [eng.sites(b) for b in range(len(np.atleast_2d(thetas)))], eng.bond_dims()


def _circuits():
    rng = np.random.default_rng(4)
    spec40, words40, coeffs40, th40 = W.batched_40q(1, batch=4, terms=800)
    yield "40q_reverse_linear", spec40["n"], spec40["ops"], words40, coeffs40, th40
    spec = O.hardware_efficient_spec(12, 3, ("ry", "rz"), "linear")
    words, coeffs = W.random_hamiltonian(rng, 12, 120, 4)
    yield "12q_linear_ryrz", 12, spec["ops"], words, coeffs, rng.uniform(-np.pi, np.pi, (3, spec["count"]))
    # non-adjacent CX (SWAP routing), custom one- and two-site matrices, trailing gates
    u = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))[0]
    u1 = np.linalg.qr(rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)))[0]
    ops = [("h", 0), ("ry", 1, 0), ("cx", 0, 3), ("u2", 2, 5, u), ("rx", 4, 1), ("cx", 5, 4),
           ("swap", 1, 6), ("u1", 3, u1), ("cx", 6, 2), ("rz", 0, 2), ("ry", 6, 3), ("s", 2), ("cx", 1, 2),
           ("ry", 3, 0, 0.5)]
    words, coeffs = W.random_hamiltonian(rng, 7, 60, 3, z_fraction=0.5)
    yield "7q_routed", 7, ops, words, coeffs, rng.uniform(-np.pi, np.pi, (2, 4))


@pytest.mark.parametrize("order", ["msb", "qubit"])
def test_pair_chain_equals_program_order_chain(vq, order):
    for name, n, ops, words, coeffs, th in _circuits():
        e1, s1, d1 = _run(vq, n, ops, words, coeffs, th, "pair", order=order)
        e0, s0, d0 = _run(vq, n, ops, words, coeffs, th, "chain", order=order)
        assert d1 == d0, name
        assert np.array_equal(e1, e0), name
        for a, b in zip(s1, s0):
            assert np.array_equal(a, b), name


def test_pair_chain_matches_oracle_and_reports_rank_guard(vq):
    spec, words, coeffs, theta = W.plain_12q(5)
    e, _, _ = _run(vq, 12, spec["ops"], words, coeffs, theta, "pair")
    ref = float(np.dot(O.expect_words(O.svd_evolve(spec, theta, 16), words).real, coeffs))
    assert abs(e[0] - ref) <= 1e-9 * max(1.0, abs(ref))
    for mode in ("pair", "chain"):
        with pytest.raises(vq.EngineError, match="insufficient"):
            _run(vq, 12, spec["ops"], words, coeffs, theta, mode, max_bond=4)


def test_pair_chain_in_partition_sets(vq):
    parts = W.uneven_partitions(seed=6, partitions=6, nmin=3, nmax=20, tmin=20, tmax=200)
    out = {}
    for mode in ("pair", "chain"):
        eng = vq.Engine(0, 16)
        eng.set_evolve_mode(mode)
        ps = eng.set_partitions([(s["n"], s["ops"], w, c) for s, w, c, _ in parts])
        out[mode] = eng.partition_energy(ps, ps.pack_theta([p[3] for p in parts], device=eng.device)).cpu().numpy()
    assert np.array_equal(out["pair"], out["chain"])
