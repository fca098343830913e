"""GPU parity of partition sets: independent circuits of uneven width and
Hamiltonian evaluated in one batch (the plain partition warm start's local
solves, independent_vqe.py:276-290, batched). Every partition must give the
oracle's energy, and exactly what a one-partition engine gives: the merged
levels run the same kernels on the same plan, so energies, per-term values,
shots and shot estimates are compared bit for bit."""
import numpy as np
import pytest
import torch
from scipy.stats import chi2

from oracle import mps_oracle as O
from oracle.workloads import random_hamiltonian, uneven_partitions

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vq(cuda_device):
    import vqemps
    return vqemps


def _small_set(seed=3, K=6):
    rng = np.random.default_rng(seed)
    parts = []
    for k in range(K):
        n = int(rng.integers(3, 15))
        T = int(rng.integers(20, 160))
        pattern = ("linear", "reverse_linear")[k % 2]
        spec = O.hardware_efficient_spec(n, 2 + k % 3, ("ry", "rz") if k % 3 == 1 else ("ry",), pattern)
        words, coeffs = random_hamiltonian(rng, n, T, 4)
        words[0] = "I" * n                      # identity word closes against the norm
        if k == 1:
            words = ["".join("Z" if c != "I" else "I" for c in w) for w in words]   # all diagonal
        x = rng.uniform(-np.pi, np.pi, spec["count"])
        parts.append((spec, words, np.asarray(coeffs), x))
    return parts


def _load(vq, eng, parts, order="msb"):
    return eng.set_partitions([(s["n"], s["ops"], w, c) for s, w, c, _ in parts], parts[0][0].get("initial"), order)


def _single(vq, spec, words, coeffs, order="msb"):
    eng = vq.Engine(0, 16)
    eng.set_spec(spec, site_order=order)
    eng.set_level_variant("dmma3_pf")
    eng.set_split_mode("off")            # partition sets run the prefix plan
    return eng, eng.set_hamiltonian(words, coeffs)


@pytest.mark.parametrize("order", ["msb", "qubit"])
def test_partition_energies_match_oracle_and_single_engine(vq, order):
    parts = _small_set()
    eng = vq.Engine(0, 16)
    ps = _load(vq, eng, parts, order)
    assert ps.K == len(parts) and ps.n_max == max(p[0]["n"] for p in parts)
    theta = ps.pack_theta([p[3] for p in parts], device=eng.device)
    e, pt = eng.partition_energy(ps, theta, per_term=True)
    e, pt = e.cpu().numpy(), pt.cpu().numpy()
    for k, (spec, words, coeffs, x) in enumerate(parts):
        ref = O.reverse_energy(spec, words, coeffs, x)
        assert abs(e[k] - ref) <= 1e-10 * max(1.0, abs(ref))
        se, sh = _single(vq, spec, words, coeffs, order)
        e1, pt1 = se.energy(sh, x, per_term=True)
        assert e1.item() == e[k]
        assert np.array_equal(pt1.cpu().numpy()[0], pt[k, :len(words)])
        assert eng.partition_bond_dims(ps, k) == se.bond_dims()


def test_copies_are_independent_parameter_sets(vq):
    parts = _small_set(seed=5, K=4)
    eng = vq.Engine(0, 16)
    ps = _load(vq, eng, parts)
    rng = np.random.default_rng(1)
    copies = 3
    thetas = [rng.uniform(-np.pi, np.pi, (copies, p[0]["count"])) for p in parts]
    e = eng.partition_energy(ps, ps.pack_theta(thetas, copies, eng.device), copies=copies).cpu().numpy()
    for k, (spec, words, coeffs, _) in enumerate(parts):
        se, sh = _single(vq, spec, words, coeffs)
        ref = se.energy(sh, thetas[k]).cpu().numpy()
        assert np.array_equal(ref, e[k * copies:(k + 1) * copies])
    # a second call with another copies count rebuilds the work lists
    e1 = eng.partition_energy(ps, ps.pack_theta([t[0] for t in thetas], 1, eng.device)).cpu().numpy()
    assert np.array_equal(e1, e[::copies])


@pytest.mark.parametrize("rng_name", ["philox", "splitmix"])
def test_partition_shots_and_estimates_equal_single_engine(vq, rng_name):
    parts = _small_set(seed=9, K=5)
    eng = vq.Engine(0, 16)
    ps = _load(vq, eng, parts)
    theta = ps.pack_theta([p[3] for p in parts], device=eng.device)
    shots, seed = 1000, 4242
    e, pt, bits = eng.partition_sampled_energy(ps, theta, shots, seed, rng_name, per_term=True, return_bits=True)
    bits2 = eng.partition_sample(ps, theta, shots, seed, rng_name)
    assert torch.equal(bits, bits2)
    for k, (spec, words, coeffs, x) in enumerate(parts):
        se, sh = _single(vq, spec, words, coeffs)
        b1 = se.sample(x, shots, seed + k, rng_name)          # state k draws with seed + k
        n = spec["n"]
        assert np.array_equal(vq.unpack_bits(b1, n)[0], vq.unpack_bits(bits[k:k + 1], ps.n_max)[0][:, :n])
        assert not vq.unpack_bits(bits[k:k + 1], ps.n_max)[0][:, n:].any()
        e1, pt1 = se.sampled_energy(sh, x, shots, seed + k, rng_name, "shared", per_term=True)
        assert e1.item() == e[k].item()
        assert np.array_equal(pt1.cpu().numpy()[0], pt[k, :len(words)].cpu().numpy())


def test_partition_philox_histogram_matches_exact_distribution(vq):
    rng = np.random.default_rng(12)
    parts = []
    for n in (4, 6, 5):
        spec = O.hardware_efficient_spec(n, 3, ("ry",), "linear")
        words, coeffs = random_hamiltonian(rng, n, 40, 3)
        parts.append((spec, words, np.asarray(coeffs), rng.uniform(-np.pi, np.pi, spec["count"])))
    eng = vq.Engine(0, 16)
    ps = _load(vq, eng, parts, "qubit")
    shots = 4096
    bits = eng.partition_sample(ps, ps.pack_theta([p[3] for p in parts], device=eng.device), shots, 31)
    arr = vq.unpack_bits(bits, ps.n_max)
    for k, (spec, _, _, x) in enumerate(parts):
        n = spec["n"]
        idx = arr[k][:, :n].astype(np.int64) @ (1 << np.arange(n - 1, -1, -1))
        obs = np.bincount(idx, minlength=1 << n)
        probs = np.abs(O.dense_statevector(spec, x)) ** 2
        keep = probs * shots > 5
        exp = probs[keep] * shots
        rest = probs[~keep].sum() * shots
        stat = np.sum((obs[keep] - exp) ** 2 / exp) + ((obs[~keep].sum() - rest) ** 2 / rest if rest > 0 else 0)
        assert stat < chi2.ppf(0.999, keep.sum())
        # the shots of partition k are also the oracle's Philox shots for seed 31 + k
        ref = O.sample_bits(O.svd_evolve(spec, x, 16), shots, 31 + k, "philox")
        assert np.array_equal(arr[k][:, :n], ref)


def test_partition_errors(vq):
    eng = vq.Engine(0, 16)
    spec = O.hardware_efficient_spec(4, 1, ("ry",), "linear")
    with pytest.raises(vq.EngineError, match="partition 1"):
        eng.set_partitions([(4, spec["ops"], ["ZZII"], [1.0]), (4, spec["ops"], ["ZQII"], [1.0])])
    with pytest.raises(vq.EngineError):
        eng.set_partitions([(1, [("ry", 0, 0)], ["Z"], [1.0])])
    ps = eng.set_partitions([(4, spec["ops"], ["ZZII"], [1.0])])
    with pytest.raises(vq.EngineError):
        eng.partition_energy(ps, torch.zeros((2, ps.P_max), dtype=torch.float64))
    eng.free_partitions(ps)
    with pytest.raises(vq.EngineError):
        eng.partition_energy(ps, torch.zeros((1, ps.P_max), dtype=torch.float64))


def test_uneven_64_partitions_full_size(vq):
    """64 partitions, n ~ U{8..48}, T ~ U{200..3000}, linear, 4 layers: the
    shot-count workload in one call; a few partitions checked against the
    oracle, all against the one-partition engine."""
    parts = uneven_partitions(seed=0)
    eng = vq.Engine(0, 16)
    ps = eng.set_partitions([(s["n"], s["ops"], w, c) for s, w, c, _ in parts])
    theta = ps.pack_theta([p[3] for p in parts], device=eng.device)
    e = eng.partition_energy(ps, theta).cpu().numpy()
    order = np.argsort([p[0]["n"] for p in parts])
    for k in (order[0], order[len(order) // 2], order[-1]):
        spec, words, coeffs, x = parts[k]
        ref = O.reverse_energy(spec, words, coeffs, x)
        assert abs(e[k] - ref) <= 1e-8 * max(1.0, abs(ref))
    for k, (spec, words, coeffs, x) in enumerate(parts):
        se, sh = _single(vq, spec, words, coeffs)
        assert se.energy(sh, x).item() == e[k]
    for shots in (1000, 4096):
        es, bits = eng.partition_sampled_energy(ps, theta, shots, 7, "philox", return_bits=True)
        es = es.cpu().numpy()
        assert np.isfinite(es).all()
        # shot noise: |E_shots - E| within 6 sigma of the per-term bound sum |c_t| / sqrt(shots)
        bound = np.array([np.abs(c).sum() for _, _, c, _ in parts]) / np.sqrt(shots)
        assert np.all(np.abs(es - e) <= 6 * bound)
        counts = vq.counts(bits, ps.n_max, 0)
        assert sum(counts.values()) == shots
