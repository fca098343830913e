"""Generate golden optimizer trajectories from the reference's own optimizers.

Runs hp-cyber/Graph-VQE's first-order SPSA (test/tools/spsa_optimizer.py) and
L-BFGS-B adapter (test/tools/lbfgs_optimizer.py), imported read-only from the
reference checkout given by REFERENCE_ROOT (default /root/reference), on fixed
analytic objectives, and writes ``optimizer_golden.json`` next to this script:
for every case the settings, the starting point, the accepted iterates (the
callback's points), the ordered evaluation log (kind and energy of every
objective, probe and calibration call, as the optimizer's metrics file records
them) and the returned result. The L-BFGS-B cases take their derivative from a
stand-in for ``reverse_mps.for_objective`` that returns the objective's exact
value and gradient, as the reference's own tests patch it
(test/tests/test_reverse_mps.py:85-110); with reverse mode 'required' every
derivative is cross-checked against one more objective call.

The reference checkout does not exist where the tests run, so the trajectories
are committed; the script is only rerun by hand.

Usage: python tests/golden/make_optimizer_golden.py
"""
from __future__ import annotations

import json
import os
import sys
import tempfile
from pathlib import Path
from unittest.mock import patch

import numpy as np

HERE = Path(__file__).resolve().parent
REFERENCE_ROOT = Path(os.environ.get("REFERENCE_ROOT", "/root/reference"))
sys.path.insert(0, str(REFERENCE_ROOT / "test" / "tools"))

import lbfgs_optimizer  # noqa: E402  (reference code)
import spsa_optimizer  # noqa: E402  (reference code)


def objective(x):
    """Smooth, non-separable test objective (values of order 10)."""
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


class _Reverse:
    engine = "analytic_stand_in"

    def value_gradient(self, x):
        return objective(x), objective_grad(x)


def _log_rows(path):
    return [json.loads(s) for s in Path(path).read_text().splitlines() if s.strip()]


def run_spsa(name, x0, env, maxiter):
    with tempfile.TemporaryDirectory() as d:
        full = dict(ANALYTIC_MPS_SPSA_METRICS=str(Path(d) / "spsa.jsonl"),
                    ANALYTIC_MPS_SPSA_STATE_DIR=str(Path(d) / "states"), **env)
        seen = []
        with patch.dict(os.environ, full):
            res = spsa_optimizer.minimize(objective, np.array(x0), callback=lambda x: seen.append(list(map(float, x))),
                                          options={"maxiter": maxiter})
        rows = _log_rows(full["ANALYTIC_MPS_SPSA_METRICS"])
    evals = [[r["event"], r["energy"]] for r in rows if r["event"] in ("objective", "gradient_probe",
                                                                        "calibration_probe")]
    cal = [r["learning_rate"] for r in rows if r["event"] == "calibration"]
    return dict(name=name, optimizer="spsa", env=env, maxiter=maxiter, x0=list(map(float, x0)), iterates=seen,
                evaluations=evals, learning_rate=cal[0] if cal else None,
                result=dict(x=list(map(float, res.x)), fun=float(res.fun), nit=int(res.nit), nfev=int(res.nfev),
                            njev=int(res.njev), success=bool(res.success), message=str(res.message)))


def run_lbfgs(name, x0, env, maxiter):
    with tempfile.TemporaryDirectory() as d:
        full = dict(ANALYTIC_MPS_LBFGS_METRICS=str(Path(d) / "lbfgs.jsonl"), ANALYTIC_MPS_LBFGS_REVERSE_MODE="required",
                    **env)
        seen = []
        with patch.dict(os.environ, full), patch("reverse_mps.for_objective", lambda fun, mode: _Reverse()):
            res = lbfgs_optimizer.minimize(objective, np.array(x0), callback=lambda x: seen.append(list(map(float, x))),
                                           options={"maxiter": maxiter})
        rows = _log_rows(full["ANALYTIC_MPS_LBFGS_METRICS"])
    evals = [[r["event"], r["energy"]] for r in rows if r["event"] in ("objective", "gradient_probe")]
    return dict(name=name, optimizer="lbfgs", env=env, maxiter=maxiter, x0=list(map(float, x0)), iterates=seen,
                evaluations=evals,
                result=dict(x=list(map(float, res.x)), fun=float(res.fun), nit=int(res.nit), nfev=int(res.nfev),
                            njev=int(res.njev), success=bool(res.success), message=str(res.message)))


def main():
    cwd = os.getcwd()
    out = []
    with tempfile.TemporaryDirectory() as work:
        os.chdir(work)            # the optimizers write state and log files relative to the working directory
        try:
            x0 = np.random.default_rng(11).uniform(-np.pi, np.pi, 9)
            out.append(run_spsa("spsa_defaults", x0, {}, 200))
            out.append(run_spsa("spsa_calibrated_no_stop", x0, dict(ANALYTIC_MPS_IMMEDIATE_ENERGY_TOL="1e-30",
                                                                     ANALYTIC_MPS_SPSA_SEED="7"), 40))
            out.append(run_spsa("spsa_fixed_rate", x0, dict(ANALYTIC_MPS_IMMEDIATE_ENERGY_TOL="1e-3",
                                                             ANALYTIC_MPS_SPSA_LEARNING_RATE="0.05",
                                                             ANALYTIC_MPS_SPSA_PERTURBATION="0.1",
                                                             ANALYTIC_MPS_SPSA_SEED="3"), 60))
            out.append(run_lbfgs("lbfgs_defaults", x0, {}, 1000))
            out.append(run_lbfgs("lbfgs_to_convergence", x0, dict(ANALYTIC_MPS_IMMEDIATE_ENERGY_TOL="1e-12"), 1000))
            out.append(run_lbfgs("lbfgs_iteration_cap", x0, dict(ANALYTIC_MPS_IMMEDIATE_ENERGY_TOL="1e-12"), 4))
        finally:
            os.chdir(cwd)
    (HERE / "optimizer_golden.json").write_text(json.dumps(out))
    for c in out:
        print(c["name"], c["result"]["nit"], c["result"]["nfev"], c["result"]["message"][:60], c["result"]["fun"])


if __name__ == "__main__":
    main()
