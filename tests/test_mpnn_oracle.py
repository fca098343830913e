"""CPU: the warm-start network's oracle is pinned by finite differences
(float64, no rounding), and the coupling-graph features / batch layout are
checked on small Hamiltonians."""
import numpy as np
import pytest

from oracle import mpnn_oracle as MO
from vqemps.mpnn import graph_features, init_params, make_batch


def _graph(seed=0, n=7):
    rng = np.random.default_rng(seed)
    from oracle.workloads import random_hamiltonian
    words, coeffs = random_hamiltonian(rng, n, 25, 3)
    node, ei, ef = graph_features(n, words, coeffs)
    return dict(node=node.astype(np.float64), src=ei[0], dst=ei[1], ef=ef.astype(np.float64))


def test_backward_matches_finite_differences():
    width, layers, out = 16, 2, 5
    flat = init_params(3, width, layers, out).astype(np.float64)
    flat += np.random.default_rng(1).normal(0, 0.05, flat.size)     # nonzero biases
    g = _graph()
    p, names = MO.unflatten(flat, width, layers, out)
    theta, cache = MO.forward(p, layers, g, bf16=False)
    dtheta = np.random.default_rng(2).normal(size=theta.shape)
    grad = MO.flatten(MO.backward(p, layers, g, cache, dtheta, bf16=False), names)
    rng = np.random.default_rng(4)
    idx = rng.choice(flat.size, 60, replace=False)
    h = 1e-6
    for i in idx:
        fp, fm = flat.copy(), flat.copy()
        fp[i] += h
        fm[i] -= h
        tp, _ = MO.forward(MO.unflatten(fp, width, layers, out)[0], layers, g, bf16=False)
        tm, _ = MO.forward(MO.unflatten(fm, width, layers, out)[0], layers, g, bf16=False)
        fd = ((tp - tm) * dtheta).sum() / (2 * h)
        assert abs(fd - grad[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, grad[i])


def test_periodic_loss_gradient_and_bf16_rounding():
    rng = np.random.default_rng(0)
    th, tg, w = rng.uniform(-3, 3, (6, 5)), rng.uniform(-3, 3, (6, 5)), rng.uniform(0.5, 2, 6)
    loss, d = MO.periodic_loss(th, tg, w)
    e = np.zeros_like(th)
    e[2, 3] = 1e-6
    fd = (MO.periodic_loss(th + e, tg, w)[0] - MO.periodic_loss(th - e, tg, w)[0]) / 2e-6
    assert abs(fd - d[2, 3]) < 1e-8
    assert MO.to_bf16(np.float32(1.0 + 2 ** -8)) == 1.0          # tie to even
    assert MO.to_bf16(np.float32(1.0 + 3 * 2 ** -8)) == 1.0 + 2 ** -6


def test_features_and_batch_layout():
    words = ["ZIII", "IZZI", "XIIX", "ZZII", "IIIZ"]
    coeffs = [2.0, -1.0, 0.5, 3.0, -4.0]
    node, ei, ef = graph_features(4, words, coeffs)
    assert node.shape == (4, 4) and np.isclose(node[0, 0], np.log1p(2.0) / 5) and np.isclose(node[3, 0], -np.log1p(4.0) / 5)
    assert np.isclose(node[0, 1], np.log1p(2.0 + 0.5 + 3.0) / 10)
    pairs = {(a, b) for a, b in ei.T}
    assert {(0, 3), (3, 0), (1, 2), (0, 1), (2, 3)} <= pairs
    k = [i for i, (a, b) in enumerate(ei.T) if (a, b) == (0, 1)][0]
    assert np.isclose(ef[k, 0], np.log1p(3.0) / 5) and ef[k, 2] == 1.0
    k3 = [i for i, (a, b) in enumerate(ei.T) if (a, b) == (3, 0)][0]
    assert np.isclose(ef[k3, 1], np.log1p(0.5) / 10) and ef[k3, 2] == 0.0 and ef[k3, 0] == 0.0
    b = make_batch([(node, ei, ef), (node, ei, ef)], "cpu")
    h = b.host
    assert b.n_nodes == 8 and b.n_edges == 2 * ei.shape[1]
    assert np.all(np.diff(h["dst"]) >= 0)
    assert np.array_equal(np.sort(h["src"][h["perm"]]), h["src"][h["perm"]])
    for i in range(8):
        assert np.all(h["dst"][h["dst_off"][i]:h["dst_off"][i + 1]] == i)
