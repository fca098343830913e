"""Drop-in for the reference's reverse-mode gradient entry points.

Mirrors test/tools/reverse_mps.py: ``register`` (:12-25) records supported
nearest-neighbour circuits, ``make_problem`` (:102-121) and ``for_objective``
(:124-139) build a problem, and ``ReverseMPS.value_gradient`` (:84-99) returns
(energy, gradient) -- here computed by the engine's adjoint kernels on the GPU
instead of torch autograd. ``MPSEnergy`` exposes the same computation as a
``torch.autograd.Function`` over a batch of parameter sets.
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import Engine

_REGISTRY = {}
_ENGINES = {}


def register(kernel, n, reps, gates, pattern, initial, param_order, pairs, final):
    """Record a supported ansatz exactly like reverse_mps.register.

    Unsupported circuits (pattern not linear/reverse_linear, reps > 6, unknown
    initial state, non-rotation gates, non-adjacent pairs) are silently not
    registered, so callers fall back as they do with the reference.
    """
    if pattern not in ("linear", "reverse_linear") or reps > 6 or initial not in (None, "0", "1", "+", "-"):
        return
    if any(not isinstance(g, str) or g.lower() not in ("rx", "ry", "rz") for g in gates):
        return
    rotations = {}
    for index, (_, q, layer, g) in enumerate(param_order):
        rotations.setdefault(layer, []).append((gates[g].lower(), q, index))
    ops = []
    for layer in range(reps + 1):
        ops.extend(rotations.get(layer, []))
        if layer < reps:
            if any(t != c + 1 for c, t in pairs[layer]):
                return
            ops.extend(("cx", c, t) for c, t in pairs[layer])
    _REGISTRY[id(kernel)] = (kernel, dict(n=n, ops=ops, initial=initial, count=len(param_order)))


def shared_engine(device: int = 0) -> Engine:
    """One engine per device and thread of use (the plugin keeps one simulator per thread)."""
    eng = _ENGINES.get(device)
    if eng is None:
        eng = Engine(device, 16)
        _ENGINES[device] = eng
    return eng


class ReverseMPS:
    """Energy and exact gradient of a registered circuit on the GPU engine.

    Same constructor and ``value_gradient`` contract as the reference class; the
    energy is the exact bond-doubling MPS energy (no SVD, no truncation).
    """
    engine = "vqemps_adjoint"

    def __init__(self, spec, words, coeffs, device=None):
        self.spec = spec
        self.words = list(words)
        self.coeffs = np.asarray(coeffs, dtype=float)
        dev = 0 if device in (None, "cuda") else (int(str(device).split(":")[1]) if ":" in str(device) else 0)
        if device == "cpu":
            raise ValueError("the B200 engine runs on CUDA devices only")
        self._eng = Engine(dev, 16)
        self._eng.set_spec(spec)
        self._ham = self._eng.set_hamiltonian(self.words, self.coeffs)

    def value_gradient(self, parameters):
        e, g = self._eng.energy_grad(self._ham, np.asarray(parameters, dtype=float))
        return float(e[0]), g[0].cpu().numpy()

    def value_gradient_batch(self, parameters):
        """(energies [B], gradients [B, P]) of a batch of parameter sets."""
        e, g = self._eng.energy_grad(self._ham, np.asarray(parameters, dtype=float))
        return e.cpu().numpy(), g.cpu().numpy()

    def energy(self, parameters):
        return self._eng.energy(self._ham, np.asarray(parameters, dtype=float)).cpu().numpy()


def make_problem(kernel, hamiltonian):
    """Problem of a registered kernel and a Hamiltonian (reverse_mps.py:102-121).

    ``hamiltonian`` may be a spin operator with ``for_each_term`` (CUDA-Q style,
    or ``vqemps.shim.SpinOperator``) or a (words, coeffs) pair indexed by qubit.
    """
    from .shim import Kernel as TapeKernel, TapeProblem
    entry = _REGISTRY.get(id(kernel))
    spec = entry[1] if entry is not None and entry[0] is kernel else None
    if spec is None and not isinstance(kernel, TapeKernel):
        return None
    width = spec["n"] if spec is not None else max(2, kernel.width)
    words, coeffs = [], []
    if isinstance(hamiltonian, tuple):
        words, coeffs = list(hamiltonian[0]), list(hamiltonian[1])
    else:
        def term(t):
            coeff = complex(t.get_coefficient())
            if abs(coeff.imag) > 1e-12:
                raise ValueError("Reverse mode requires Hermitian real Pauli coefficients")
            word = t.to_string(False).strip().ljust(width, "I")
            if len(word) != width or any(p not in "IXYZ" for p in word):
                raise ValueError("Unsupported Pauli encoding")
            words.append(word)
            coeffs.append(coeff.real)
        if hasattr(hamiltonian, "for_each_term"):
            hamiltonian.for_each_term(term)
        else:
            term(hamiltonian)
    if spec is None:
        return TapeProblem(kernel, words, coeffs)
    return ReverseMPS(spec, words, coeffs)


def for_objective(fun, mode):
    """Reverse problem of an objective (reverse_mps.py:124-139)."""
    if mode == "off":
        return None
    if mode not in ("auto", "hybrid", "required"):
        raise ValueError("Reverse mode must be off, auto, hybrid or required")
    factory = getattr(fun, "reverse_factory", None)
    if factory is not None:
        return factory()
    pair = getattr(fun, "reverse_problem", None)
    owner = getattr(fun, "__self__", None)
    names = ("CUDAQVQE", "SHARCVQE", "CVaRVQE")
    if (pair is None and owner is not None and type(owner).__name__ in names
            and getattr(fun, "__name__", "") == "cost_func"):
        if type(owner).__name__ == "CVaRVQE" and owner.alpha != 1.0:
            raise ValueError("Reverse CVaR requires alpha=1")
        pair = (owner.kernel, owner.hamiltonian)
    return make_problem(*pair) if pair is not None else None


class MPSEnergy(torch.autograd.Function):
    """E(theta) for a batch [B, P] of parameter sets; backward uses the adjoint kernels.

    ``MPSEnergy.apply(theta, engine, ham)`` returns the B energies. When autograd
    will need dE/dtheta (grad mode on and ``theta`` requiring grad) the forward
    pass runs the adjoint sweep once and keeps the gradient for the backward
    pass; otherwise (under ``torch.no_grad()``, or for a ``theta`` that needs no
    gradient) it runs the energy-only path, about a third of the cost.
    """

    @classmethod
    def apply(cls, theta, engine, ham):
        # grad mode is always off inside forward(), so it is read here
        need = bool(torch.is_grad_enabled() and getattr(theta, "requires_grad", False))
        return super().apply(theta, engine, ham, need)

    @staticmethod
    def forward(ctx, theta, engine, ham, need_grad):
        th = theta.detach().to(device=engine.device, dtype=torch.float64).contiguous()
        if th.dim() == 1:
            th = th.unsqueeze(0)
        if need_grad:
            e, g = engine.energy_grad(ham, th)
            ctx.save_for_backward(g)
        else:
            e = engine.energy(ham, th)
        ctx.squeeze = theta.dim() == 1
        out = e.to(theta.device)
        return out[0] if ctx.squeeze else out

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        go = grad_out.to(g.device, torch.float64)
        if ctx.squeeze:
            return (go * g[0]).to(grad_out.device), None, None, None
        return (go[:, None] * g).to(grad_out.device), None, None, None


def mps_energy(theta, engine, ham):
    return MPSEnergy.apply(theta, engine, ham)
