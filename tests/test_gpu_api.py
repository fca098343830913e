"""The reference-facing entry points on the GPU engine: CUDA-Q-shaped
observe/observe_async/sample, the ReverseMPS-compatible gradient problems and
the torch.autograd.Function, each against the oracle (FP64: 1e-9 relative for
energies, 1e-8 of the largest component for gradients)."""
import math

import numpy as np
import pytest
import torch

from oracle import mps_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api(cuda_device):
    from vqemps import reverse, shim
    return shim, reverse


def build_ansatz(shim, n, reps, gates=("ry", "rz"), pattern="linear"):
    count = n * (reps + 1) * len(gates)
    kernel, *theta = shim.make_kernel(*([float] * count))
    q = kernel.qalloc(n)
    index = 0
    for layer in range(reps + 1):
        for k in range(n):
            for g in gates:
                getattr(kernel, g)(theta[index], q[k])
                index += 1
        if layer < reps:
            for a, b in O.pairs_for_pattern(n, layer, pattern):
                kernel.cx(q[a], q[b])
    return kernel, O.hardware_efficient_spec(n, reps, gates, pattern)


def test_observe_matches_oracle_and_async(api):
    shim, _ = api
    kernel, spec = build_ansatz(shim, 6, 2)
    x = np.random.default_rng(0).uniform(-np.pi, np.pi, spec["count"])
    H = 0.4 * shim.spin.z(0) - 0.7 * shim.spin.z(1) * shim.spin.z(2) + 0.2 * shim.spin.x(3) * shim.spin.y(5) + 0.9
    words, coeffs = H.words(6)
    ref = float(np.dot(O.dense_expectations(O.dense_statevector(spec, x), words).real, np.real(coeffs)))
    e = shim.observe(kernel, H, *x, shots_count=-1).expectation()
    assert abs(e - ref) < 1e-9 * max(1, abs(ref))
    e2 = shim.observe_async(kernel, H, *x, qpu_id=0).get().expectation()
    assert e2 == e
    r = shim.observe(kernel, H, *x)
    sub = shim.spin.z(1) * shim.spin.z(2)
    psi = O.dense_statevector(spec, x)
    assert abs(r.expectation(sub) - O.dense_expectations(psi, ["IZZIII"])[0].real) < 1e-10


def test_observe_async_overlaps_kernels_and_keeps_each_result(api):
    """Several observe_async calls are queued before any get(): on two kernels
    (two engines) and twice on the same kernel, whose second submission first
    finishes the first one. Each result equals the synchronous observe."""
    shim, _ = api
    k1, spec1 = build_ansatz(shim, 6, 2)
    k2, spec2 = build_ansatz(shim, 8, 3, pattern="reverse_linear")
    rng = np.random.default_rng(5)
    x1 = rng.uniform(-np.pi, np.pi, spec1["count"])
    x2 = rng.uniform(-np.pi, np.pi, spec2["count"])
    H1 = 0.4 * shim.spin.z(0) - 0.7 * shim.spin.z(1) * shim.spin.z(2) + 0.2 * shim.spin.x(3) * shim.spin.y(5)
    H2 = 1.3 * shim.spin.z(7) * shim.spin.z(0) - 0.5 * shim.spin.x(4) + 0.25
    ref1 = shim.observe(k1, H1, *x1).expectation()
    ref1b = shim.observe(k1, H1, *(-x1)).expectation()
    ref2 = shim.observe(k2, H2, *x2).expectation()
    a = shim.observe_async(k1, H1, *x1, qpu_id=0)
    b = shim.observe_async(k2, H2, *x2, qpu_id=1)
    c = shim.observe_async(k1, H1, *(-x1), qpu_id=0)
    assert c.get().expectation() == ref1b
    assert b.get().expectation() == ref2
    assert a.get().expectation() == ref1
    assert a.done() and b.done() and c.done()


def test_known_answer_two_qubits_through_the_shim(api):
    shim, _ = api
    kernel, theta = shim.make_kernel(float)
    q = kernel.qalloc(2)
    kernel.ry(theta, q[0])
    kernel.x(q[1])
    kernel.cx(q[0], q[1])
    paulis = (shim.spin.i(0), shim.spin.z(0), shim.spin.z(1), shim.spin.x(0) * shim.spin.x(1),
              shim.spin.y(0) * shim.spin.y(1), shim.spin.z(0) * shim.spin.z(1), shim.spin.x(1))
    H = 0.11 * paulis[0]
    for index, p in enumerate(paulis[1:], start=1):
        H = H + (0.11 + 0.03 * index) * p
    t = 0.37
    e = shim.observe(kernel, H, t, shots_count=-1).expectation()
    assert abs(e - (-0.15 + 0.43 * math.sin(t) - 0.03 * math.cos(t))) < 1e-10
    diag = 0.17 * shim.spin.i(0) + 0.23 * shim.spin.z(0) - 0.31 * shim.spin.z(1) + 0.19 * shim.spin.z(0) * shim.spin.z(1)
    assert math.isfinite(shim.observe(kernel, diag, t, shots_count=4096).expectation())
    counts = shim.sample(kernel, t, shots_count=4096)
    assert sum(counts.values()) == 4096
    assert all(len(k) == 2 for k in counts)


def test_sample_keys_put_qubit_zero_left(api):
    shim, _ = api
    kernel = shim.make_kernel()
    q = kernel.qalloc(7)
    kernel.x(q[0])
    counts = shim.sample(kernel, shots_count=100)
    assert counts == {"1000000": 100}


def test_tape_problem_gradient_with_affine_angles(api):
    shim, reverse = api
    kernel, a, b = shim.make_kernel(float, float)
    q = kernel.qalloc(3)
    kernel.ry(2 * a + 0.3, q[0])
    kernel.cx(q[0], q[1])
    kernel.rz(b - a, q[1])
    kernel.rx(0.5 * b, q[2])
    kernel.cx(q[1], q[2])
    H = shim.spin.z(0) * shim.spin.x(1) + 0.3 * shim.spin.y(2) - 0.8 * shim.spin.z(1) * shim.spin.z(2)
    prob = reverse.make_problem(kernel, H)
    x = np.array([0.4, -1.2])
    e, g = prob.value_gradient(x)
    h = 1e-5
    f = lambda v: shim.observe(kernel, H, *v).expectation()
    fd = np.array([(f(x + h * d) - f(x - h * d)) / (2 * h) for d in np.eye(2)])
    assert abs(e - f(x)) < 1e-10
    np.testing.assert_allclose(g, fd, atol=1e-7)


def test_register_make_problem_for_objective(api):
    _, reverse = api
    n, reps = 4, 2
    order = [(f"t{layer}_{q}_{g}", q, layer, g) for layer in range(reps + 1) for q in range(n) for g in range(2)]
    k = object()
    reverse.register(k, n, reps, ("ry", "rz"), "reverse_linear", None, order,
                     [[(i, i + 1) for i in range(n - 2, -1, -1)]] * reps, True)
    words, coeffs = ["ZZII", "IXYI", "IIIZ"], [0.5, -0.25, 1.5]
    prob = reverse.make_problem(k, (words, coeffs))
    spec = reverse._REGISTRY[id(k)][1]
    x = np.random.default_rng(1).normal(size=len(order))
    e, g = prob.value_gradient(x)
    eref, gref = O.reverse_value_gradient(spec, words, coeffs, x)
    assert abs(e - eref) < 1e-10
    np.testing.assert_allclose(g, gref, atol=1e-10)
    bad = object()
    reverse.register(bad, 3, 9, ("ry",), "linear", None, [], [], [])
    assert id(bad) not in reverse._REGISTRY
    assert reverse.for_objective(lambda v: sum(v), "auto") is None
    fun = lambda v: 0.0
    fun.reverse_problem = (k, (words, coeffs))
    assert abs(reverse.for_objective(fun, "required").value_gradient(x)[0] - eref) < 1e-10


def test_autograd_function_backward(api):
    _, reverse = api
    import vqemps
    spec = O.hardware_efficient_spec(5, 2, ("ry",), "linear")
    words, coeffs = ["ZIIII", "IZZII", "IIXIX", "YIIIY"], np.array([1.0, -0.5, 0.25, 0.75])
    eng = vqemps.Engine(0, 16)
    eng.set_spec(spec)
    ham = eng.set_hamiltonian(words, coeffs)
    th = torch.tensor(np.random.default_rng(2).normal(size=(3, spec["count"])), dtype=torch.float64,
                      requires_grad=True)
    e = reverse.mps_energy(th, eng, ham)
    w = torch.tensor([1.0, -2.0, 0.5], dtype=torch.float64)
    (e * w).sum().backward()
    for b in range(3):
        eref, gref = O.reverse_value_gradient(spec, words, coeffs, th.detach().numpy()[b])
        assert abs(float(e[b].detach()) - eref) < 1e-10
        np.testing.assert_allclose(th.grad[b].numpy(), w[b].item() * gref, atol=1e-10)
