"""CUDA-graph capture of engine calls: a replay equals the direct call bit for
bit, and follows new angles written into the captured theta tensor."""
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


def test_captured_energy_replays_bitwise(vq):
    spec, words, coeffs, x = W.plain_12q(seed=1)
    eng = vq.Engine(0, 16)
    eng.set_spec(spec)
    ham = eng.set_hamiltonian(words, coeffs)
    rng = np.random.default_rng(0)
    th = torch.tensor(rng.uniform(-np.pi, np.pi, (4, spec["count"])), device=eng.device)
    out = torch.empty(4, dtype=torch.float64, device=eng.device)
    g = eng.capture(lambda: eng.energy(ham, th, out=out, check_status=False))
    for _ in range(3):
        new = rng.uniform(-np.pi, np.pi, (4, spec["count"]))
        th.copy_(torch.from_numpy(new))
        g.replay()
        torch.cuda.synchronize()
        direct = eng.energy(ham, torch.from_numpy(new).to(eng.device))
        assert torch.equal(out, direct)
        ref = O.reverse_energy(spec, words, coeffs, new[0])
        assert abs(out[0].item() - ref) <= 1e-10 * max(1.0, abs(ref))


def test_captured_partition_energy_replays_bitwise(vq):
    parts = W.uneven_partitions(seed=2, partitions=5, nmin=4, nmax=14, tmin=20, tmax=200)
    eng = vq.Engine(0, 16)
    ps = eng.set_partitions([(s["n"], s["ops"], w, c) for s, w, c, _ in parts])
    theta = ps.pack_theta([p[3] for p in parts], device=eng.device)
    out = torch.empty(ps.K, dtype=torch.float64, device=eng.device)
    g = eng.capture(lambda: eng.partition_energy(ps, theta, out=out, check_status=False))
    theta.mul_(0.5)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(out, eng.partition_energy(ps, theta))


@pytest.mark.parametrize("split", [True, False])
def test_captured_split_real_levels_replay_bitwise(vq, split):
    """40 qubits, real-arithmetic levels; with the split evaluation (per-term cuts,
    environments kept in per-level regions) the suffix half runs on the engine's
    second stream, forked from and joined into the captured stream: replays equal
    direct calls bit for bit."""
    from vqemps import workloads as VW
    spec, words, coeffs, thetas = VW.batched_40q(seed=3, batch=8, terms=1500)
    eng = vq.Engine(0, 16)
    eng.set_split_mode(split)
    eng.set_spec(spec)
    eng.set_level_variant("real_pf")
    ham = eng.set_hamiltonian(words, coeffs)
    assert (eng.plan_stats(ham)["cut"] >= 0) == split
    th = torch.tensor(thetas, device=eng.device)
    out = torch.empty(8, dtype=torch.float64, device=eng.device)
    g = eng.capture(lambda: eng.energy(ham, th, out=out, check_status=False))
    rng = np.random.default_rng(5)
    for _ in range(2):
        new = thetas + rng.normal(scale=0.05, size=thetas.shape)
        th.copy_(torch.from_numpy(new))
        g.replay()
        torch.cuda.synchronize()
        direct = eng.energy(ham, torch.from_numpy(new).to(eng.device))
        assert torch.equal(out, direct)
    eng.close()
