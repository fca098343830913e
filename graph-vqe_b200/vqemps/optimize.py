"""Optimizer drivers over batched engine calls.

``spsa_minimize`` is the reference's first-order SPSA (test/tools/spsa_optimizer.py:
settings :42-55, perturbation_gradient :58-63, calibration :129-138, update loop
:142-176, immediate energy stop :169-173) with its evaluations batched: the five
calibration pairs are one call of B = 10, and every update evaluates the
candidate together with the NEXT update's two probes (B = 3). The Rademacher
draws happen in the reference's order from the same ``default_rng(seed)``, and
no draw depends on an energy, so the iterates equal the sequential algorithm's
for equal energies.

``lbfgs_minimize`` is the reference's L-BFGS-B adapter
(test/tools/lbfgs_optimizer.py:57-208) with the reverse derivative coming from
the same engine call as the energy: one ``energy_grad`` per point serves both
the objective and the derivative, so the reference's extra probe observe
(:132-143) is not needed; its one-time cross-check against the objective can be
kept with ``check_energy``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from scipy.optimize import OptimizeResult
from scipy.optimize import minimize as scipy_minimize


@dataclass
class SpsaSettings:
    """Defaults of spsa_optimizer.settings() (ANALYTIC_MPS_SPSA_* unset)."""
    perturbation: float = 0.2
    learning_rate: float | None = None      # None: calibrate
    alpha: float = 0.602
    gamma: float = 0.101
    stability: float = 0.0
    calibration_pairs: int = 5
    target_update: float = 2 * np.pi / 10
    seed: int = 0
    immediate_energy_tol: float | None = 1.0

    def validate(self):
        for key in ("perturbation", "alpha", "gamma", "target_update"):
            v = getattr(self, key)
            if not np.isfinite(v) or v <= 0:
                raise ValueError(f"Invalid SPSA {key}")
        if not np.isfinite(self.stability) or self.stability < 0:
            raise ValueError("Invalid SPSA stability")
        if self.learning_rate is not None and (not np.isfinite(self.learning_rate) or self.learning_rate <= 0):
            raise ValueError("Invalid SPSA learning rate")
        if self.calibration_pairs < 1:
            raise ValueError("SPSA calibration_pairs must be positive")


def _bounds_arrays(bounds, size):
    if bounds is None:
        return np.full(size, -np.inf), np.full(size, np.inf)
    if hasattr(bounds, "lb"):
        return np.broadcast_to(bounds.lb, (size,)).astype(float), np.broadcast_to(bounds.ub, (size,)).astype(float)
    lo = np.array([-np.inf if b[0] is None else b[0] for b in bounds], dtype=float)
    hi = np.array([np.inf if b[1] is None else b[1] for b in bounds], dtype=float)
    return lo, hi


def spsa_minimize(energies, x0, maxiter: int = 1000, settings: SpsaSettings | None = None, bounds=None,
                  callback=None):
    """SPSA on ``energies(X) -> E`` (X: [B, P] angles, E: [B]) with batched probes.

    Returns an OptimizeResult with the reference's fields (best x and energy,
    nit, nfev counted per parameter set, njev, message) plus ``calls``: the
    number of batched energy calls.
    """
    cfg = settings or SpsaSettings()
    cfg.validate()
    if maxiter < 1:
        raise ValueError("Positive SPSA iteration cap required")
    x = np.asarray(x0, dtype=float).copy()
    if x.ndim != 1 or not np.isfinite(x).all():
        raise ValueError("Expected finite one-dimensional initial parameters")
    lower, upper = _bounds_arrays(bounds, x.size)
    if np.any(lower > upper):
        raise ValueError("Invalid bounds")
    x = np.clip(x, lower, upper)
    rng = np.random.default_rng(cfg.seed)
    counts = dict(objective=0, gradient_probe=0, calibration_probe=0, gradient=0, accepted_iteration=0, calls=0)

    def run(points):
        e = np.asarray(energies(np.asarray(points, dtype=float)), dtype=float).reshape(-1)
        counts["calls"] += 1
        if not np.isfinite(e).all():
            raise ValueError(f"Nonfinite SPSA energy: {e}")
        return e

    def rademacher():
        return rng.choice(np.array([-1.0, 1.0]), size=x.size)

    a = cfg.learning_rate
    c = cfg.perturbation
    if not x.size:
        fx = float(run(x[None, :])[0])
        return OptimizeResult(x=x, fun=fx, nit=0, nfev=1, njev=0, success=True,
                              message="No variational parameters", calls=counts["calls"])
    # objective at x0, then the calibration pairs (all in one call)
    pts = [x]
    deltas = []
    if a is None:
        for _ in range(cfg.calibration_pairs):
            d = rademacher()
            deltas.append(d)
            pts += [x + c * d, x - c * d]
    # first update's probes (they depend only on x and the next draws)
    k = 1
    ck = c / k ** cfg.gamma
    d_next = rademacher()
    pts += [x + ck * d_next, x - ck * d_next]
    e = run(pts)
    fx = float(e[0])
    counts["objective"] += 1
    best_x, best_f = x.copy(), fx
    if a is None:
        mags = []
        for i, d in enumerate(deltas):
            plus, minus = e[1 + 2 * i], e[2 + 2 * i]
            mags.append(float(np.mean(np.abs(((plus - minus) / (2 * c)) * d))))
        counts["calibration_probe"] += 2 * len(deltas)
        magnitude = float(np.mean(mags))
        a = cfg.target_update * (cfg.stability + 1) ** cfg.alpha / magnitude if magnitude > 1e-12 else 1.0
    probes = e[-2:]
    status = "SPSA iteration cap reached"
    nit = 0
    for k in range(1, maxiter + 1):
        previous = fx
        ak = a / (k + cfg.stability) ** cfg.alpha
        ck = c / k ** cfg.gamma
        g = ((probes[0] - probes[1]) / (2 * ck)) * d_next
        counts["gradient_probe"] += 2
        counts["gradient"] += 1
        candidate = np.clip(x - ak * g, lower, upper)
        pts = [candidate]
        if k < maxiter:
            ck1 = c / (k + 1) ** cfg.gamma
            d_next = rademacher()
            pts += [candidate + ck1 * d_next, candidate - ck1 * d_next]
        e = run(pts)
        fx = float(e[0])
        counts["objective"] += 1
        probes = e[1:]
        x = candidate
        nit = k
        counts["accepted_iteration"] += 1
        if fx < best_f:
            best_x, best_f = x.copy(), fx
        if callback is not None:
            callback(x)
        tol = cfg.immediate_energy_tol
        if tol is not None and abs(fx - previous) < tol:
            status = f"Immediate energy stopping: |delta E| < {tol}; no patience/window"
            break
    nfev = counts["objective"] + counts["gradient_probe"] + counts["calibration_probe"]
    return OptimizeResult(x=best_x, fun=best_f, nit=nit, nfev=nfev, njev=counts["gradient"],
                          success=status.startswith("Immediate energy"), message=status, calls=counts["calls"],
                          learning_rate=a)


class ImmediateEnergyStop(Exception):
    pass


@dataclass
class _ValueGradCache:
    fn: object
    x: np.ndarray | None = None
    value: float = 0.0
    grad: np.ndarray | None = None
    calls: int = 0

    def get(self, x):
        x = np.asarray(x, dtype=float)
        if self.x is None or not np.array_equal(x, self.x):
            v, g = self.fn(x)
            self.calls += 1
            self.x, self.value, self.grad = x.copy(), float(v), np.asarray(g, dtype=float).copy()
        return self.value, self.grad


def lbfgs_minimize(value_grad, x0, bounds=None, maxiter: int = 1000000, ftol: float = 1e-9, gtol: float = 1e-3,
                   immediate_energy_tol: float | None = 1.0, energy=None, check_energy: bool = False,
                   callback=None, maxls: int = 40, maxcor: int = 10):
    """L-BFGS-B on ``value_grad(x) -> (E, dE/dx)`` (the reverse derivative).

    Defaults are the reference adapter's (ANALYTIC_MPS_LBFGS_FTOL 1e-9, _GTOL 1e-3,
    maxls 40, maxcor 10, immediate energy stop 1.0 between consecutive
    objective values). ``check_energy`` compares the first reverse energy with
    ``energy(x)`` (the objective) at rtol 1e-9 / atol 1e-7 like the adapter's
    auto mode and raises on a mismatch.
    """
    x0 = np.asarray(x0, dtype=float)
    if hasattr(bounds, "lb"):
        bounds = list(zip(bounds.lb, bounds.ub))
    cache = _ValueGradCache(value_grad)
    best = [float("inf"), x0.copy()]
    previous = [None]
    counts = dict(objective=0, gradient=0, accepted_iteration=0)
    checked = [not check_energy]

    def fun(x):
        v, _ = cache.get(x)
        counts["objective"] += 1
        if not np.isfinite(v):
            raise ValueError(f"Nonfinite objective energy: {v}")
        if v < best[0]:
            best[:] = [v, np.asarray(x, dtype=float).copy()]
        delta = None if previous[0] is None else abs(v - previous[0])
        previous[0] = v
        if immediate_energy_tol is not None and delta is not None and delta < immediate_energy_tol:
            raise ImmediateEnergyStop()
        return v

    def jac(x):
        v, g = cache.get(x)
        counts["gradient"] += 1
        if not checked[0]:
            observed = float(energy(np.asarray(x, dtype=float)))
            if not np.isclose(v, observed, rtol=1e-9, atol=1e-7):
                raise RuntimeError(f"Reverse energy {v} differs from the objective {observed}")
            checked[0] = True
        return g

    def accepted(xk):
        counts["accepted_iteration"] += 1
        if callback is not None:
            callback(xk)

    if not x0.size:
        v, _ = cache.get(x0)
        return OptimizeResult(x=x0, fun=v, nit=0, nfev=1, njev=0, success=True,
                              message="No variational parameters", engine_calls=cache.calls)
    try:
        res = scipy_minimize(fun, x0, method="L-BFGS-B", jac=jac, bounds=bounds, callback=accepted,
                             options=dict(maxiter=maxiter, maxfun=maxiter, ftol=ftol, gtol=gtol, maxls=maxls,
                                          maxcor=maxcor))
        res.engine_calls = cache.calls
        res.best_energy = best[0]
        return res
    except ImmediateEnergyStop:
        tol = immediate_energy_tol
        return OptimizeResult(x=best[1], fun=best[0], nfev=counts["objective"], njev=counts["gradient"],
                              nit=counts["accepted_iteration"], success=True, engine_calls=cache.calls,
                              message=f"Immediate energy stopping: consecutive |delta E| < {tol:g} "
                                      "(no patience/window)")
