"""The optimizer drivers over the GPU engine at the benchmark's size (40 qubits,
5,000 terms): batched SPSA issues its calibration pairs and probes as batches
and still equals the sequential algorithm evaluated one parameter set per call;
L-BFGS-B over the adjoint gradient cross-checks every reverse energy against the
SVD-path objective (rtol 1e-9, the reference adapter's 'required' mode); the
batched line search evaluates its step lengths four per call."""
import numpy as np
import pytest
import torch

from oracle import optim_oracle as OO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem(cuda_device):
    import vqemps
    from vqemps import workloads as W
    spec, words, coeffs, thetas = W.batched_40q(seed=0, batch=2)
    eng = vqemps.Engine(0, 16)
    eng.set_spec(spec)
    eng.set_level_variant("dmma3_pf")       # one kernel for every batch size: bitwise equal energies
    ham = eng.set_hamiltonian(words, coeffs)
    yield vqemps, spec, words, coeffs, thetas, eng, ham
    eng.close()


def test_spsa_over_engine_batches_and_equals_sequential(problem):
    from vqemps.optimize import SpsaSettings, spsa_minimize
    vq, spec, words, coeffs, thetas, eng, ham = problem

    def energies(X):
        return eng.energy(ham, torch.tensor(np.atleast_2d(X), device=eng.device)).cpu().numpy()

    sizes, seen = [], []
    res = spsa_minimize(energies, thetas[0], maxiter=4, settings=SpsaSettings(immediate_energy_tol=None, seed=2),
                        call_sizes=sizes, callback=lambda x: seen.append(x.copy()))
    assert sizes == [13, 3, 3, 3, 1]          # x0 + 5 calibration pairs + first probes, then candidate + probes
    bx, bf, nit, nfev, traj = OO.spsa_sequential(lambda x: float(energies(x)[0]), thetas[0], 4, seed=2,
                                                 immediate_energy_tol=None)
    assert res.nit == nit == 4 and res.nfev == nfev
    assert res.fun == bf and np.array_equal(res.x, bx)
    assert all(np.array_equal(a, b) for a, b in zip(seen, traj))


def test_lbfgs_over_adjoint_gradient_checks_every_energy(problem):
    from vqemps.optimize import lbfgs_minimize
    from vqemps.reverse import ReverseMPS
    vq, spec, words, coeffs, thetas, eng, ham = problem
    rev = ReverseMPS(spec, words, coeffs)
    trace = []
    objective = lambda x: float(eng.energy(ham, torch.tensor(x[None], device=eng.device))[0])  # noqa: E731
    res = lbfgs_minimize(rev.value_gradient, thetas[1], maxiter=6, immediate_energy_tol=None, energy=objective,
                         check_energy="every", trace=trace)
    probes = [v for k, v in trace if k == "gradient_probe"]
    objectives = [v for k, v in trace if k == "objective"]
    assert len(probes) == res.njev >= 2
    assert res.fun < objectives[0]
    with pytest.raises(RuntimeError, match="differs from the objective"):
        lbfgs_minimize(rev.value_gradient, thetas[1], maxiter=2, immediate_energy_tol=None,
                       energy=lambda x: objective(x) + 1e-3, check_energy="every")


def test_batched_line_search_over_engine(problem):
    from vqemps.optimize import lbfgs_minimize
    from vqemps.reverse import ReverseMPS
    vq, spec, words, coeffs, thetas, eng, ham = problem
    rev = ReverseMPS(spec, words, coeffs)
    accepted = []
    res = lbfgs_minimize(None, thetas[0], maxiter=6, immediate_energy_tol=None, line_search="batched",
                         value_grad_batch=rev.value_gradient_batch, candidates=4,
                         callback=lambda x: accepted.append(float(rev.value_gradient(x)[0])))
    assert res.nit >= 1 and res.call_sizes[0] == 1 and all(s == 4 for s in res.call_sizes[1:])
    e0 = rev.value_gradient(thetas[0])[0]
    assert all(b < a for a, b in zip([e0] + accepted, accepted))       # every accepted step decreases E
    assert res.fun == min(accepted)
