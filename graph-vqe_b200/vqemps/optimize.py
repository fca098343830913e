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
the objective and the derivative. The adapter's cross-check of the reverse
energy against the objective (:132-143) is ``check_energy``: "every" derivative
(reverse mode 'required'), the "first" one (mode 'auto') or never. Its stop
rules are the adapter's immediate stop on consecutive objective values
(``immediate_energy_tol``) and the strategy's stop on the improvement of an
accepted iterate (``accepted_energy_tol``, independent_vqe.py:210-223).
``line_search="batched"`` replaces scipy's sequential line search by a
backtracking search that evaluates several step lengths in ONE engine call.

``cobyla_minimize`` is the strategy's COBYLA solve (independent_vqe.py:236-241)
with the same accepted-iterate stop.

Every driver can append its evaluations to ``trace`` as [kind, energy] pairs
in the order the sequential reference makes them (kinds "objective",
"gradient_probe", "calibration_probe"), which is how the tests compare them
with the reference's own evaluation logs.
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
                  callback=None, trace: list | None = None, call_sizes: list | None = None):
    """SPSA on ``energies(X) -> E`` (X: [B, P] angles, E: [B]) with batched probes.

    Returns an OptimizeResult with the reference's fields (best x and energy,
    nit, nfev counted per parameter set, njev, message) plus ``calls``: the
    number of batched energy calls. ``call_sizes`` (a list) receives the batch
    size of every call.
    """
    log = trace.append if trace is not None else (lambda item: None)
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
        if call_sizes is not None:
            call_sizes.append(len(points))
        if not np.isfinite(e).all():
            raise ValueError(f"Nonfinite SPSA energy: {e}")
        return e

    def rademacher():
        return rng.choice(np.array([-1.0, 1.0]), size=x.size)

    a = cfg.learning_rate
    c = cfg.perturbation
    if not x.size:
        fx = float(run(x[None, :])[0])
        log(["objective", fx])
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
    log(["objective", fx])
    for v in e[1:1 + 2 * len(deltas)]:
        log(["calibration_probe", float(v)])
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
        log(["gradient_probe", float(probes[0])])
        log(["gradient_probe", float(probes[1])])
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
        log(["objective", fx])
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


def _check_mode(check_energy):
    if check_energy is True:
        return "first"
    if check_energy in (False, None):
        return None
    if check_energy not in ("first", "every"):
        raise ValueError(f"check_energy must be False, 'first' or 'every', not {check_energy!r}")
    return check_energy


def lbfgs_minimize(value_grad, x0, bounds=None, maxiter: int = 1000000, ftol: float = 1e-9, gtol: float = 1e-3,
                   immediate_energy_tol: float | None = 1.0, energy=None, check_energy=False,
                   callback=None, maxls: int = 40, maxcor: int = 10, accepted_energy_tol: float | None = None,
                   trace: list | None = None, line_search: str = "scipy", value_grad_batch=None,
                   candidates: int = 4):
    """L-BFGS-B on ``value_grad(x) -> (E, dE/dx)`` (the reverse derivative).

    Defaults are the reference adapter's (ANALYTIC_MPS_LBFGS_FTOL 1e-9, _GTOL 1e-3,
    maxls 40, maxcor 10, immediate energy stop 1.0 between consecutive
    objective values). ``check_energy`` ("first", "every" or False; True means
    "first") compares the reverse energy with ``energy(x)`` (the objective) at
    rtol 1e-9 / atol 1e-7 like the adapter's auto / required modes and raises
    on a mismatch. ``accepted_energy_tol`` stops as soon as an accepted iterate
    improves the energy by less than it (the strategy's callback rule).

    ``line_search="batched"`` runs :func:`lbfgs_batched` instead (unbounded
    problems only): ``value_grad_batch(X) -> (E[B], G[B, P])`` then evaluates
    ``candidates`` step lengths per engine call.
    """
    if line_search == "batched":
        if bounds is not None:
            raise ValueError("the batched line search does not take bounds")
        if value_grad_batch is None:
            def value_grad_batch(X):
                out = [value_grad(x) for x in np.atleast_2d(X)]
                return np.array([o[0] for o in out]), np.array([o[1] for o in out])
        return lbfgs_batched(value_grad_batch, x0, maxiter=maxiter, gtol=gtol, ftol=ftol, maxcor=maxcor,
                             candidates=candidates, immediate_energy_tol=immediate_energy_tol,
                             accepted_energy_tol=accepted_energy_tol, callback=callback, trace=trace)
    if line_search != "scipy":
        raise ValueError(f"unknown line search {line_search!r}")
    x0 = np.asarray(x0, dtype=float)
    if hasattr(bounds, "lb"):
        bounds = list(zip(bounds.lb, bounds.ub))
    log = trace.append if trace is not None else (lambda item: None)
    mode = _check_mode(check_energy)
    if mode is not None and energy is None:
        raise ValueError("check_energy needs the objective `energy`")
    cache = _ValueGradCache(value_grad)
    best = [float("inf"), x0.copy()]
    previous = [None]
    accepted_prev = [None]
    counts = dict(objective=0, gradient=0, accepted_iteration=0)
    checked = [mode is None]
    reason = [None]

    def fun(x):
        v, _ = cache.get(x)
        counts["objective"] += 1
        log(["objective", v])
        if not np.isfinite(v):
            raise ValueError(f"Nonfinite objective energy: {v}")
        if accepted_prev[0] is None:
            accepted_prev[0] = v
        if v < best[0]:
            best[:] = [v, np.asarray(x, dtype=float).copy()]
        delta = None if previous[0] is None else abs(v - previous[0])
        previous[0] = v
        if immediate_energy_tol is not None and delta is not None and delta < immediate_energy_tol:
            reason[0] = (f"Immediate energy stopping: consecutive |delta E| < {immediate_energy_tol:g} "
                         "(no patience/window)")
            raise ImmediateEnergyStop()
        return v

    def jac(x):
        v, g = cache.get(x)
        counts["gradient"] += 1
        if mode == "every" or not checked[0]:
            observed = float(energy(np.asarray(x, dtype=float)))
            log(["gradient_probe", observed])
            if not np.isclose(v, observed, rtol=1e-9, atol=1e-7):
                raise RuntimeError(f"Reverse energy {v} differs from the objective {observed}")
            checked[0] = True
        return g

    def accepted(xk):
        counts["accepted_iteration"] += 1
        if callback is not None:
            callback(xk)
        if accepted_energy_tol is not None:
            v, _ = cache.get(xk)
            improvement = accepted_prev[0] - v
            accepted_prev[0] = v
            if improvement < accepted_energy_tol:
                reason[0] = "energy_improvement_below_threshold"
                raise ImmediateEnergyStop()

    if not x0.size:
        v, _ = cache.get(x0)
        log(["objective", v])
        return OptimizeResult(x=x0, fun=v, nit=0, nfev=1, njev=0, success=True,
                              message="No variational parameters", engine_calls=cache.calls)
    try:
        res = scipy_minimize(fun, x0, method="L-BFGS-B", jac=jac, bounds=bounds, callback=accepted,
                             options=dict(maxiter=maxiter, maxfun=maxiter, ftol=ftol, gtol=gtol, maxls=maxls,
                                          maxcor=maxcor))
        res.engine_calls = cache.calls
        res.best_energy = best[0]
        res.best_x = best[1]
        return res
    except ImmediateEnergyStop:
        return OptimizeResult(x=best[1], fun=best[0], nfev=counts["objective"], njev=counts["gradient"],
                              nit=counts["accepted_iteration"], success=True, engine_calls=cache.calls,
                              best_energy=best[0], best_x=best[1], message=reason[0])


def lbfgs_batched(value_grad_batch, x0, maxiter: int = 1000, gtol: float = 1e-3, ftol: float = 1e-9,
                  maxcor: int = 10, candidates: int = 4, shrink: float = 0.5, c1: float = 1e-4, c2: float = 0.9,
                  immediate_energy_tol: float | None = None, accepted_energy_tol: float | None = None,
                  callback=None, trace: list | None = None, max_rounds: int = 10):
    """L-BFGS whose line search evaluates several step lengths in one call.

    The direction is the standard two-loop L-BFGS direction (memory ``maxcor``);
    the first step of the first iteration is scaled to a unit move. Each line
    search round evaluates ``candidates`` step lengths alpha, alpha * shrink,
    ... in ONE ``value_grad_batch`` call (energies and gradients of all of them)
    and accepts the longest that satisfies the weak Wolfe conditions
    (sufficient decrease c1, curvature c2), else the longest with sufficient
    decrease, else it continues below the shortest. A batched engine evaluates
    a few parameter sets for about the price of one (the calls are latency
    bound), so a backtracking search costs one call instead of several.

    Stops: projected-gradient norm (max abs) <= gtol; relative decrease below
    ftol (scipy's rule); ``immediate_energy_tol`` on consecutive objective
    values; ``accepted_energy_tol`` on the improvement of an accepted iterate;
    ``maxiter`` iterations. Returns an OptimizeResult (best point) with
    ``engine_calls`` and ``call_sizes``.
    """
    log = trace.append if trace is not None else (lambda item: None)
    x = np.asarray(x0, dtype=float).copy()
    sizes = []

    def run(X):
        e, g = value_grad_batch(np.asarray(X, dtype=float))
        e = np.asarray(e, dtype=float).reshape(-1)
        g = np.asarray(g, dtype=float).reshape(len(e), -1)
        sizes.append(len(e))
        if not np.isfinite(e).all() or not np.isfinite(g).all():
            raise ValueError("Nonfinite energy or gradient in the line search")
        return e, g

    e0, g0 = run(x[None, :])
    f, g = float(e0[0]), g0[0]
    log(["objective", f])
    best = [f, x.copy()]
    S, Y = [], []
    nit = 0
    message = "STOP: TOTAL NO. OF ITERATIONS REACHED LIMIT"
    previous = f
    if np.max(np.abs(g)) <= gtol:
        return OptimizeResult(x=x, fun=f, nit=0, nfev=1, njev=1, success=True,
                              message="CONVERGENCE: NORM OF PROJECTED GRADIENT <= PGTOL", engine_calls=1,
                              call_sizes=sizes)
    nfev = 1
    for it in range(maxiter):
        # two-loop recursion
        q = g.copy()
        alphas = []
        for s_, y_ in reversed(list(zip(S, Y))):
            rho = 1.0 / float(y_ @ s_)
            a_ = rho * float(s_ @ q)
            alphas.append((rho, a_))
            q -= a_ * y_
        if S:
            q *= float(S[-1] @ Y[-1]) / float(Y[-1] @ Y[-1])
        for (s_, y_), (rho, a_) in zip(zip(S, Y), reversed(alphas)):
            b_ = rho * float(y_ @ q)
            q += (a_ - b_) * s_
        d = -q
        slope = float(g @ d)
        if slope >= 0:                       # not a descent direction: restart from steepest descent
            S.clear(); Y.clear()
            d = -g
            slope = float(g @ d)
        alpha = 1.0 if S else min(1.0, 1.0 / max(np.linalg.norm(d), 1e-300))
        chosen = None
        for _ in range(max_rounds):
            steps = alpha * shrink ** np.arange(candidates)
            E, G = run(x[None, :] + steps[:, None] * d[None, :])
            nfev += len(steps)
            armijo = E <= f + c1 * steps * slope
            wolfe = armijo & (G @ d >= c2 * slope)
            pick = np.flatnonzero(wolfe)
            if not len(pick):
                pick = np.flatnonzero(armijo)
            if len(pick):
                j = int(pick[0])
                chosen = (steps[j], float(E[j]), G[j])
                break
            alpha = steps[-1] * shrink
        if chosen is None:
            message = "ABNORMAL_TERMINATION_IN_LNSRCH"
            break
        step, f_new, g_new = chosen
        s_vec = step * d
        y_vec = g_new - g
        if float(s_vec @ y_vec) > 1e-10 * float(y_vec @ y_vec):
            S.append(s_vec); Y.append(y_vec)
            if len(S) > maxcor:
                S.pop(0); Y.pop(0)
        x = x + s_vec
        f_old, f, g = f, f_new, g_new
        nit = it + 1
        log(["objective", f])
        if f < best[0]:
            best = [f, x.copy()]
        if callback is not None:
            callback(x)
        if immediate_energy_tol is not None and abs(f - previous) < immediate_energy_tol:
            message = (f"Immediate energy stopping: consecutive |delta E| < {immediate_energy_tol:g} "
                       "(no patience/window)")
            break
        if accepted_energy_tol is not None and (previous - f) < accepted_energy_tol:
            message = "energy_improvement_below_threshold"
            break
        previous = f
        if np.max(np.abs(g)) <= gtol:
            message = "CONVERGENCE: NORM OF PROJECTED GRADIENT <= PGTOL"
            break
        if (f_old - f) / max(abs(f_old), abs(f), 1.0) <= ftol:
            message = "CONVERGENCE: REL_REDUCTION_OF_F_<=_FACTR*EPSMCH"
            break
    return OptimizeResult(x=best[1], fun=best[0], nit=nit, nfev=nfev, njev=nfev, message=message,
                          success=not message.startswith(("ABNORMAL", "STOP")), engine_calls=len(sizes),
                          call_sizes=sizes)


def cobyla_minimize(energy, x0, maxiter: int, tol: float = 1e-8, accepted_energy_tol: float | None = None,
                    callback=None, trace: list | None = None):
    """COBYLA on ``energy(x)`` (the strategy's non-gradient solve,
    independent_vqe.py:236-241) with the accepted-iterate stop."""
    log = trace.append if trace is not None else (lambda item: None)
    x0 = np.asarray(x0, dtype=float)
    cache = {}
    best = [float("inf"), x0.copy()]
    prev = [None]
    counts = dict(objective=0, accepted_iteration=0)

    def fun(x):
        key = np.asarray(x, dtype=float).tobytes()
        if key not in cache:
            v = float(energy(np.asarray(x, dtype=float)))
            cache[key] = v
            counts["objective"] += 1
            log(["objective", v])
            if prev[0] is None:
                prev[0] = v
            if v < best[0]:
                best[:] = [v, np.asarray(x, dtype=float).copy()]
        return cache[key]

    def accepted(xk, *_, **__):
        xk = np.asarray(xk, dtype=float)
        counts["accepted_iteration"] += 1
        v = fun(xk)
        if callback is not None:
            callback(xk)
        if accepted_energy_tol is not None:
            improvement = prev[0] - v
            prev[0] = v
            cache.clear()
            cache[xk.tobytes()] = v
            if improvement < accepted_energy_tol:
                raise ImmediateEnergyStop()

    fun(x0)
    try:
        res = scipy_minimize(fun, x0, method="COBYLA", callback=accepted, options=dict(maxiter=maxiter, tol=tol))
        message = str(res.message)
    except ImmediateEnergyStop:
        message = "energy_improvement_below_threshold"
    return OptimizeResult(x=best[1], fun=best[0], nit=counts["accepted_iteration"], nfev=counts["objective"],
                          message=message, success=True)
