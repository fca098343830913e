"""Optimizer drivers (CPU): batched SPSA equals the reference's sequential SPSA
(restated in the oracle) iterate for iterate; the L-BFGS-B adapter keeps the
reference's defaults and immediate energy stop."""
import numpy as np
import pytest

from oracle import optim_oracle as OO
from vqemps.optimize import SpsaSettings, lbfgs_minimize, spsa_minimize


def _objective(x):
    x = np.atleast_2d(x)
    return 3.0 * np.sum(np.sin(x) ** 2, axis=1) + 0.5 * np.sum(np.cos(2 * x[:, :1] - x[:, -1:]), axis=1)


@pytest.mark.parametrize("tol,maxiter", [(None, 25), (1e-3, 200)])
@pytest.mark.parametrize("lr", [None, 0.05])
def test_batched_spsa_equals_sequential(tol, maxiter, lr):
    x0 = np.random.default_rng(3).uniform(-np.pi, np.pi, 11)
    seen = []
    res = spsa_minimize(lambda X: _objective(X), x0, maxiter=maxiter,
                        settings=SpsaSettings(learning_rate=lr, immediate_energy_tol=tol, seed=5),
                        callback=lambda x: seen.append(x.copy()))
    bx, bf, nit, nfev, traj = OO.spsa_sequential(lambda x: _objective(x)[0], x0, maxiter, learning_rate=lr,
                                                 immediate_energy_tol=tol, seed=5)
    assert res.nit == nit and res.nfev == nfev
    assert res.fun == bf and np.array_equal(res.x, bx)
    assert len(seen) == len(traj) and all(np.array_equal(a, b) for a, b in zip(seen, traj))
    # one call for x0 + calibration + first probes, then one per update
    assert res.calls == 1 + nit


def test_spsa_bounds_and_validation():
    with pytest.raises(ValueError):
        spsa_minimize(lambda X: _objective(X), np.zeros(3), settings=SpsaSettings(perturbation=-1))
    res = spsa_minimize(lambda X: _objective(X), np.full(4, 3.0), maxiter=20,
                        settings=SpsaSettings(immediate_energy_tol=None), bounds=[(-1, 1)] * 4)
    assert np.all(np.abs(res.x) <= 1)


def test_lbfgs_adapter_matches_scipy_and_stops_early():
    from scipy.optimize import minimize, rosen, rosen_der
    x0 = np.array([-1.2, 1.0, 0.3])
    ref = minimize(rosen, x0, jac=rosen_der, method="L-BFGS-B",
                   options=dict(ftol=1e-9, gtol=1e-3, maxls=40, maxcor=10))
    got = lbfgs_minimize(lambda x: (rosen(x), rosen_der(x)), x0, immediate_energy_tol=None)
    assert np.array_equal(got.x, ref.x) and got.nit == ref.nit
    assert got.engine_calls <= ref.nfev          # one engine call serves objective and derivative
    stopped = lbfgs_minimize(lambda x: (rosen(x), rosen_der(x)), x0, immediate_energy_tol=1.0)
    assert stopped.message.startswith("Immediate energy stopping")
    with pytest.raises(RuntimeError):
        lbfgs_minimize(lambda x: (rosen(x), rosen_der(x)), x0, energy=lambda x: rosen(x) + 1.0,
                       check_energy=True, immediate_energy_tol=None)
