"""GPU: the warm-start network's hand-written forward, backward, loss and Adam
kernels against the numpy oracle with the same BF16 operand rounding."""
import numpy as np
import pytest
import torch

from oracle import mpnn_oracle as MO
from oracle.workloads import random_hamiltonian

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mp(cuda_device):
    from vqemps import mpnn
    return mpnn


def _graphs(mp, sizes=(6, 9, 12), seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for n in sizes:
        words, coeffs = random_hamiltonian(rng, n, 8 * n, 4)
        out.append(mp.graph_features(n, words, coeffs))
    return out


def _host_graph(batch):
    h = batch.host
    return dict(node=h["node"].astype(np.float64), src=h["src"], dst=h["dst"], ef=h["ef"].astype(np.float64))


def _relerr(a, b):
    return np.linalg.norm(np.asarray(a, float) - np.asarray(b, float)) / max(np.linalg.norm(b), 1e-30)


def test_forward_backward_match_oracle(mp):
    net = mp.MPNN(0, params=None, seed=5)
    flat = net.params().astype(np.float64)
    flat[np.abs(flat) < 1e-12] = 0.01          # nonzero biases
    net.set_params(flat.astype(np.float32))
    flat = net.params().astype(np.float64)
    batch = mp.make_batch(_graphs(mp), net.device)
    theta = net.forward(batch).cpu().numpy()
    p, names = MO.unflatten(flat)
    g = _host_graph(batch)
    ref, cache = MO.forward(p, 3, g, bf16=True)
    assert theta.shape == ref.shape
    assert _relerr(theta, ref) < 2e-3
    rng = np.random.default_rng(1)
    dtheta = rng.normal(size=theta.shape).astype(np.float32)
    grad = net.backward(batch, torch.tensor(dtheta, device=net.device)).cpu().numpy().copy()
    ref_g = MO.backward(p, 3, g, cache, dtheta.astype(np.float64), bf16=True)
    o = 0
    for name in names:
        size = ref_g[name].size
        assert _relerr(grad[o:o + size], ref_g[name].reshape(-1)) < 1e-2, name
        o += size
    # deterministic: the same backward again is bitwise equal
    again = net.backward(batch, torch.tensor(dtheta, device=net.device)).cpu().numpy()
    assert np.array_equal(grad, again)


def test_loss_and_adam_match_oracle(mp):
    net = mp.MPNN(0, seed=2)
    batch = mp.make_batch(_graphs(mp, (5, 7)), net.device)
    theta = net.forward(batch)
    rng = np.random.default_rng(3)
    target = torch.tensor(rng.uniform(-3, 3, theta.shape), dtype=torch.float32, device=net.device)
    weight = torch.tensor(rng.uniform(0.5, 2.0, theta.shape[0]), dtype=torch.float32, device=net.device)
    loss, dtheta = net.loss(target, weight)
    ref_l, ref_d = MO.periodic_loss(theta.cpu().numpy().astype(np.float64), target.cpu().numpy(),
                                    weight.cpu().numpy())
    assert abs(loss.item() - ref_l) < 1e-5 * max(1, abs(ref_l))
    assert np.allclose(dtheta.cpu().numpy(), ref_d, atol=1e-7)
    w0 = net.params().astype(np.float64)
    grad = net.backward(batch, dtheta).cpu().numpy().astype(np.float64)
    net.adam(lr=1e-2)
    w_ref, _, _ = MO.adam(w0, grad, np.zeros_like(w0), np.zeros_like(w0), 1, 1e-2)
    assert np.allclose(net.params(), w_ref, atol=1e-6)


def test_training_fits_a_teacher(mp):
    teacher = mp.MPNN(0, seed=11)
    student = mp.MPNN(0, seed=12)
    graphs = _graphs(mp, (8, 10, 12, 14), seed=7)
    batch = mp.make_batch(graphs, teacher.device)
    target = teacher.forward(batch).clone()
    first = None
    for step in range(300):
        loss = student.train_step(batch, target, lr=2e-3).item()
        first = loss if first is None else first
    assert loss < 0.25 * first
