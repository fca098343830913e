"""The optimizer drivers against the reference's own SPSA and L-BFGS-B
(tests/golden/optimizer_golden.json, written by make_optimizer_golden.py, which
runs test/tools/spsa_optimizer.py and lbfgs_optimizer.py on fixed analytic
objectives). Iterates, results and the ordered evaluation logs must be equal
bit for bit; the oracle's sequential SPSA restatement is pinned the same way."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import optim_oracle as OO
from vqemps.optimize import SpsaSettings, lbfgs_minimize, spsa_minimize

GOLDEN = json.loads((Path(__file__).parent / "golden" / "optimizer_golden.json").read_text())


def objective(x):
    x = np.asarray(x, dtype=float)
    return float(3.0 * np.sum(np.sin(x) ** 2) + 0.5 * np.cos(2 * x[0] - x[-1]) + 0.25 * np.sum(x[:-1] * x[1:]))


def objective_grad(x):
    x = np.asarray(x, dtype=float)
    g = 3.0 * np.sin(2 * x)
    s = np.sin(2 * x[0] - x[-1])
    g[0] += -1.0 * s
    g[-1] += 0.5 * s
    g[:-1] += 0.25 * x[1:]
    g[1:] += 0.25 * x[:-1]
    return g


def _spsa_settings(env):
    lr = env.get("ANALYTIC_MPS_SPSA_LEARNING_RATE", "auto")
    return SpsaSettings(perturbation=float(env.get("ANALYTIC_MPS_SPSA_PERTURBATION", "0.2")),
                        learning_rate=None if lr == "auto" else float(lr),
                        seed=int(env.get("ANALYTIC_MPS_SPSA_SEED", "0")),
                        immediate_energy_tol=float(env.get("ANALYTIC_MPS_IMMEDIATE_ENERGY_TOL", "1")))


def _same_result(res, g):
    assert list(map(float, res.x)) == g["x"]
    assert float(res.fun) == g["fun"]
    assert (int(res.nit), int(res.nfev), int(res.njev)) == (g["nit"], g["nfev"], g["njev"])
    assert str(res.message) == g["message"] and bool(res.success) == g["success"]


@pytest.mark.parametrize("case", [c for c in GOLDEN if c["optimizer"] == "spsa"], ids=lambda c: c["name"])
def test_batched_spsa_equals_reference_spsa(case):
    seen, trace, sizes = [], [], []
    res = spsa_minimize(lambda X: np.array([objective(x) for x in X]), np.array(case["x0"]),
                        maxiter=case["maxiter"], settings=_spsa_settings(case["env"]),
                        callback=lambda x: seen.append(list(map(float, x))), trace=trace, call_sizes=sizes)
    assert seen == case["iterates"]
    assert trace == case["evaluations"]
    _same_result(res, case["result"])
    if case["learning_rate"] is not None:
        assert res.learning_rate == case["learning_rate"]
    # one call holds the objective, the calibration pairs and the first probes; then 3 per update
    pairs = 5 if case["learning_rate"] is not None else 0
    assert sizes[0] == 1 + 2 * pairs + 2 and all(s == 3 for s in sizes[1:-1]) and sizes[-1] in (1, 3)


@pytest.mark.parametrize("case", [c for c in GOLDEN if c["optimizer"] == "spsa"], ids=lambda c: c["name"])
def test_oracle_spsa_restatement_equals_reference(case):
    cfg = _spsa_settings(case["env"])
    bx, bf, nit, nfev, traj = OO.spsa_sequential(objective, np.array(case["x0"]), case["maxiter"],
                                                 perturbation=cfg.perturbation, learning_rate=cfg.learning_rate,
                                                 seed=cfg.seed, immediate_energy_tol=cfg.immediate_energy_tol)
    assert [list(map(float, t)) for t in traj] == case["iterates"]
    assert list(map(float, bx)) == case["result"]["x"] and bf == case["result"]["fun"]
    assert (nit, nfev) == (case["result"]["nit"], case["result"]["nfev"])


@pytest.mark.parametrize("case", [c for c in GOLDEN if c["optimizer"] == "lbfgs"], ids=lambda c: c["name"])
def test_lbfgs_adapter_equals_reference_lbfgs(case):
    """Reverse mode 'required': every derivative is cross-checked against one more
    objective call, which appears in the log as a gradient probe."""
    seen, trace = [], []
    tol = float(case["env"].get("ANALYTIC_MPS_IMMEDIATE_ENERGY_TOL", "1"))
    res = lbfgs_minimize(lambda x: (objective(x), objective_grad(x)), np.array(case["x0"]),
                         maxiter=case["maxiter"], immediate_energy_tol=tol, energy=objective, check_energy="every",
                         callback=lambda x: seen.append(list(map(float, x))), trace=trace)
    assert seen == case["iterates"]
    assert trace == case["evaluations"]
    _same_result(res, case["result"])


def test_batched_line_search_converges_with_fewer_calls():
    """The batched line search reaches the same minimum as scipy's L-BFGS-B on
    Rosenbrock, with its step lengths evaluated a few at a time."""
    from scipy.optimize import rosen, rosen_der

    def batch(X):
        X = np.atleast_2d(X)
        return np.array([rosen(x) for x in X]), np.array([rosen_der(x) for x in X])

    x0 = np.array([-1.2, 1.0, 0.3, -0.5])
    ref = lbfgs_minimize(lambda x: (rosen(x), rosen_der(x)), x0, immediate_energy_tol=None, gtol=1e-8, ftol=1e-14)
    got = lbfgs_minimize(None, x0, immediate_energy_tol=None, gtol=1e-8, ftol=1e-14, line_search="batched",
                         value_grad_batch=batch, candidates=4)
    assert got.success and np.allclose(got.x, ref.x, atol=1e-5) and got.fun < 1e-10
    assert max(got.call_sizes) == 4 and got.engine_calls < ref.engine_calls
    with pytest.raises(ValueError):
        lbfgs_minimize(None, x0, bounds=[(-2, 2)] * 4, line_search="batched", value_grad_batch=batch)
