"""CPU: angle layouts of the learned warm start and its canonical training
target (a product state with the solve's magnetizations)."""
import numpy as np

from oracle import mps_oracle as O
from vqemps.warmstart import angles_to_theta, canonical_angles, theta_to_angles
from vqemps.workloads import ansatz_spec, warm_start_problem


def test_angle_layout_round_trip_and_wrap():
    n = 7
    theta = np.random.default_rng(0).uniform(-9, 9, 5 * n)
    ang = theta_to_angles(theta, n)
    assert ang.shape == (n, 5) and np.all(ang <= np.pi) and np.all(ang > -np.pi)
    back = angles_to_theta(ang)
    assert np.allclose(np.cos(back), np.cos(theta)) and np.allclose(np.sin(back), np.sin(theta))
    assert ang[3, 2] == theta_to_angles(theta, n)[3, 2]
    assert np.isclose(np.cos(ang[3, 2]), np.cos(theta[2 * n + 3]))     # layer 2, qubit 3


def test_canonical_target_reproduces_magnetizations():
    n = 5
    mag = np.array([1.0, -1.0, 0.3, -0.7, 0.0])
    theta = angles_to_theta(canonical_angles(mag))
    spec = ansatz_spec(n)
    psi = O.dense_statevector(spec, theta)
    words = ["I" * q + "Z" + "I" * (n - q - 1) for q in range(n)]
    assert np.allclose(O.dense_expectations(psi, words).real, mag, atol=1e-12)


def test_training_problems_are_seeded():
    a, b = warm_start_problem(5), warm_start_problem(5)
    assert a[0] == b[0] and a[1] == b[1] and np.array_equal(a[2], b[2])
    assert 16 <= a[0] <= 48 and len(a[1]) == 25 * a[0]
