"""CUDA-Q-shaped front end of the engine: the observe/sample/gradient entry points
that the reference's VQE driver and optimizers call.

Reference call shapes (test/sources/independent-vqe/Qiskit_VQE/subspace_vqe.py:583-585,
test/tools/analytic_execution.py:67-80, sampled_execution.py:35-47,
test/tools/run_case.py:107-108):

  kernel, *theta = make_kernel(float, float, ...);  q = kernel.qalloc(n)
  kernel.ry(theta[i], q[k]); kernel.cx(q[a], q[b]) ...
  observe(kernel, H, *values, shots_count=-1).expectation()
  observe_async(kernel, H, *values, qpu_id=0).get().expectation()
  sample(kernel, *values, shots_count=1000).items()      # keys: qubit 0 leftmost

The kernel records its gate tape like test/tools/circuit_tape.py (parameter
expressions included); angles are affine functions of the kernel arguments and
are evaluated on the host, the state is prepared and measured by the engine.
Shot seeds follow the plugin: sampleSeed starts at 1234567 and increments per
shot-based call (simulator_mps_dist.cu:214,1495,1601).
"""
from __future__ import annotations

import threading
from concurrent.futures import Future

import numpy as np
import torch

from .engine import Engine, counts as _counts

_lock = threading.Lock()
_state = dict(sample_seed=1234567, max_bond=16)


def set_random_seed(seed: int):
    _state["sample_seed"] = int(seed)


# ---------------------------------------------------------------------------
# parameters, qubits, kernels
# ---------------------------------------------------------------------------
class Parameter:
    """Affine expression sum_i a_i theta_i + b of kernel arguments."""

    def __init__(self, coef=None, const=0.0):
        self.coef = dict(coef or {})
        self.const = float(const)

    @staticmethod
    def of(v):
        return v if isinstance(v, Parameter) else Parameter({}, float(v))

    def __add__(self, o):
        o = Parameter.of(o)
        c = dict(self.coef)
        for k, v in o.coef.items():
            c[k] = c.get(k, 0.0) + v
        return Parameter(c, self.const + o.const)

    __radd__ = __add__

    def __neg__(self):
        return Parameter({k: -v for k, v in self.coef.items()}, -self.const)

    def __sub__(self, o):
        return self + (-Parameter.of(o))

    def __rsub__(self, o):
        return Parameter.of(o) + (-self)

    def __mul__(self, o):
        if isinstance(o, Parameter):
            if o.coef and self.coef:
                raise TypeError("angles must be affine in the kernel arguments")
            if not o.coef:
                o = o.const
            else:
                return o * self
        return Parameter({k: v * o for k, v in self.coef.items()}, self.const * o)

    __rmul__ = __mul__

    def __truediv__(self, o):
        if isinstance(o, Parameter):
            if o.coef:
                raise TypeError("angles must be affine in the kernel arguments")
            o = o.const
        return self * (1.0 / o)


class Qubit:
    def __init__(self, index):
        self.index = int(index)


class Kernel:
    """Gate tape of one kernel; the engine program is compiled lazily."""

    def __init__(self, nparams):
        self.parameters = [Parameter({i: 1.0}) for i in range(nparams)]
        self.width = 0
        self.operations = []          # (name, qubits, Parameter | None)
        self._program = None

    def qalloc(self, count):
        if self.width:
            raise ValueError("one register allocation per kernel")
        if int(count) < 2:
            raise RuntimeError("the MPS engine needs >= 2 qubits")
        self.width = int(count)
        return [Qubit(i) for i in range(count)]

    def compile(self):
        self.program()

    def _rot(self, name):
        def op(angle, qubit):
            self.operations.append((name, (qubit.index,), Parameter.of(angle)))
            self._program = None
        return op

    def __getattr__(self, name):
        if name in ("rx", "ry", "rz"):
            return self._rot(name)
        if name in ("h", "x", "y", "z", "s", "sdg", "cx", "swap"):
            def gate(*qubits):
                self.operations.append((name, tuple(q.index for q in qubits), None))
                self._program = None
            return gate
        raise AttributeError(f"unsupported kernel operation: {name}")

    def program(self):
        """Engine op list with one angle slot per rotation, and the affine map
        angles = A @ args + b from kernel arguments to slots."""
        if self._program is None:
            ops, rows, consts = [], [], []
            for name, qs, expr in self.operations:
                if name in ("rx", "ry", "rz"):
                    ops.append((name, qs[0], len(rows)))
                    rows.append(expr.coef)
                    consts.append(expr.const)
                else:
                    ops.append((name, *qs))
            A = np.zeros((len(rows), len(self.parameters)))
            for r, coef in enumerate(rows):
                for k, v in coef.items():
                    A[r, k] = v
            self._program = (ops, A, np.asarray(consts, dtype=float))
        return self._program

    def angles(self, args):
        _, A, b = self.program()
        x = np.asarray(args, dtype=float).reshape(-1, len(self.parameters)) if len(self.parameters) else \
            np.zeros((1, 0))
        return x @ A.T + b



def make_kernel(*types):
    if any(t is not float for t in types):
        raise TypeError("kernel arguments must be scalar floats")
    k = Kernel(len(types))
    return (k, *k.parameters) if types else k


# ---------------------------------------------------------------------------
# spin operators (qubit-indexed Pauli words, q0 first)
# ---------------------------------------------------------------------------
_PMUL = {("I", p): (1, p) for p in "IXYZ"}
_PMUL.update({(p, "I"): (1, p) for p in "IXYZ"})
_PMUL.update({(p, p): (1, "I") for p in "XYZ"})
_PMUL.update({("X", "Y"): (1j, "Z"), ("Y", "X"): (-1j, "Z"), ("Y", "Z"): (1j, "X"),
              ("Z", "Y"): (-1j, "X"), ("Z", "X"): (1j, "Y"), ("X", "Z"): (-1j, "Y")})


class Term:
    def __init__(self, word, coeff):
        self.word, self.coeff = word, coeff

    def get_coefficient(self):
        return self.coeff

    def to_string(self, with_coefficient=True):
        return self.word if not with_coefficient else f"{self.coeff} {self.word}"


class SpinOperator:
    def __init__(self, terms=None):
        self.terms = dict(terms or {})      # word (tuple of (q, P)) -> complex coeff

    @staticmethod
    def single(q, p):
        return SpinOperator({((q, p),) if p != "I" else (): 1.0})

    def _width(self):
        qs = [q for w in self.terms for q, _ in w]
        return max(qs) + 1 if qs else 1

    def __add__(self, o):
        if not isinstance(o, SpinOperator):
            o = SpinOperator({(): complex(o)})
        t = dict(self.terms)
        for k, v in o.terms.items():
            t[k] = t.get(k, 0) + v
        return SpinOperator(t)

    __radd__ = __add__

    def __neg__(self):
        return SpinOperator({k: -v for k, v in self.terms.items()})

    def __sub__(self, o):
        return self + (-o if isinstance(o, SpinOperator) else -complex(o))

    def __mul__(self, o):
        if not isinstance(o, SpinOperator):
            return SpinOperator({k: v * o for k, v in self.terms.items()})
        out = {}
        for w1, c1 in self.terms.items():
            for w2, c2 in o.terms.items():
                d = dict(w1)
                ph = 1
                for q, p in w2:
                    f, r = _PMUL[(d.get(q, "I"), p)]
                    ph *= f
                    if r == "I":
                        d.pop(q, None)
                    else:
                        d[q] = r
                key = tuple(sorted(d.items()))
                out[key] = out.get(key, 0) + c1 * c2 * ph
        return SpinOperator(out)

    def __rmul__(self, o):
        return self * o

    def words(self, width=None):
        width = width or self._width()
        ws, cs = [], []
        for w, c in self.terms.items():
            chars = ["I"] * width
            for q, p in w:
                chars[q] = p
            ws.append("".join(chars))
            cs.append(c)
        return ws, cs

    def for_each_term(self, fn):
        ws, cs = self.words()
        for w, c in zip(ws, cs):
            fn(Term(w, c))

    def get_term_count(self):
        return len(self.terms)

    def __iter__(self):
        ws, cs = self.words()
        return iter([Term(w, c) for w, c in zip(ws, cs)])


class _Spin:
    @staticmethod
    def i(q): return SpinOperator.single(q, "I")

    @staticmethod
    def x(q): return SpinOperator.single(q, "X")

    @staticmethod
    def y(q): return SpinOperator.single(q, "Y")

    @staticmethod
    def z(q): return SpinOperator.single(q, "Z")


spin = _Spin()


# ---------------------------------------------------------------------------
# results
# ---------------------------------------------------------------------------
class ObserveResult:
    def __init__(self, energy, words, values):
        self._energy = float(energy)
        self._values = dict(zip(words, values))

    def expectation(self, sub=None):
        if sub is None:
            return self._energy
        width = len(next(iter(self._values))) if self._values else 1
        ws, cs = sub.words(width)
        return float(sum((c * self._values[w]).real for w, c in zip(ws, cs)))


class SampleResult(dict):
    def count(self, key):
        return self.get(key, 0)

    def most_probable(self):
        return max(self, key=self.get)


# ---------------------------------------------------------------------------
# execution
# ---------------------------------------------------------------------------
class _Runner:
    """Engines and loaded Hamiltonians cached per kernel (one engine per width)."""

    def __init__(self):
        self.engines = {}
        self.hams = {}

    def engine(self, kernel):
        key = id(kernel)
        ent = self.engines.get(key)
        prog = kernel.program()
        if ent is None or ent[1] is not prog:
            eng = ent[0] if ent is not None else Engine(0, _state["max_bond"])
            eng.set_circuit(max(2, kernel.width), prog[0], site_order="msb")
            self.engines[key] = (eng, prog)
            self.hams = {k: v for k, v in self.hams.items() if k[0] != key}
        return self.engines[key][0]

    def ham(self, kernel, eng, H):
        width = max(2, kernel.width)
        ws, cs = H.words(width)
        if any(abs(complex(c).imag) > 1e-12 for c in cs):
            raise ValueError("Hamiltonian must have real Pauli coefficients")
        key = (id(kernel), tuple(ws), tuple(complex(c).real for c in cs))
        h = self.hams.get(key)
        if h is None:
            h = eng.set_hamiltonian(ws, [complex(c).real for c in cs])
            self.hams[key] = h
        return h, ws


_runner = _Runner()


def _next_seed():
    with _lock:
        s = _state["sample_seed"]
        _state["sample_seed"] = s + 1
    return s


class AsyncObserveResult:
    """An observe call whose kernels are queued on the engine's stream.

    ``get()`` waits for them, checks the state's status and returns the
    ObserveResult. The engine keeps one status word per state, which the next
    call on the same engine overwrites, so submitting another call on that
    engine first finishes this one (its result or error is kept for ``get()``);
    calls on other kernels' engines overlap freely."""

    def __init__(self, eng, ws, e, pt):
        self._eng, self._ws, self._e, self._pt = eng, ws, e, pt
        self._event = torch.cuda.Event()
        self._event.record(torch.cuda.current_stream(eng.device))
        self._future = None

    def done(self):
        return self._future is not None or self._event.query()

    def _finish(self):
        if self._future is not None:
            return
        f = Future()
        try:
            self._event.synchronize()
            self._eng.check_status(1)
            f.set_result(ObserveResult(float(self._e[0]), self._ws, self._pt[0].cpu().numpy()))
        except BaseException as exc:      # kept for get(), as a Future does
            f.set_exception(exc)
        self._future = f
        if _pending.get(id(self._eng)) is self:
            del _pending[id(self._eng)]

    def get(self):
        self._finish()
        return self._future.result()


_pending = {}


def _submit(kernel, hamiltonian, args, shots_count):
    eng = _runner.engine(kernel)
    prev = _pending.get(id(eng))
    if prev is not None:
        prev._finish()
    h, ws = _runner.ham(kernel, eng, hamiltonian)
    ang = kernel.angles(args)
    if shots_count is None or shots_count < 0:
        e, pt = eng.energy(h, ang, per_term=True, check_status=False)
    else:
        e, pt = eng.sampled_energy(h, ang, int(shots_count), _next_seed(), "splitmix", "plugin", per_term=True,
                                   check_status=False)
    res = AsyncObserveResult(eng, ws, e, pt)
    _pending[id(eng)] = res
    return res


def observe(kernel, hamiltonian, *args, shots_count=-1, qpu_id=0, noise_model=None, **_):
    if noise_model is not None:
        raise RuntimeError("noise models are not supported by the MPS engine")
    return _submit(kernel, hamiltonian, args, shots_count).get()


def observe_async(kernel, hamiltonian, *args, shots_count=-1, qpu_id=0, noise_model=None, **_):
    """Queue the evaluation and return at once; ``.get()`` waits for it."""
    if noise_model is not None:
        raise RuntimeError("noise models are not supported by the MPS engine")
    return _submit(kernel, hamiltonian, args, shots_count)


def sample(kernel, *args, shots_count=1000, **_):
    eng = _runner.engine(kernel)
    ang = kernel.angles(args)
    bits = eng.sample(ang, int(shots_count), _next_seed(), "splitmix")
    return SampleResult(_counts(bits, kernel.width))


class TapeProblem:
    """Energy and gradient of a recorded kernel (the reference's recorded_problem /
    ReverseTapeMPS route, reverse_mps.py:141-215): the adjoint kernels give
    dE/d(angle slot), the affine angle map gives dE/d(argument) = A^T g."""
    engine = "vqemps_adjoint_tape"

    def __init__(self, kernel, words, coeffs):
        self.kernel = kernel
        self.eng = Engine(0, _state["max_bond"])
        ops, self.A, self.b = kernel.program()
        self.eng.set_circuit(max(2, kernel.width), ops, site_order="msb")
        self.ham = self.eng.set_hamiltonian(list(words), np.asarray(coeffs, dtype=float))

    def value_gradient(self, parameters):
        ang = self.kernel.angles(parameters)
        e, g = self.eng.energy_grad(self.ham, ang)
        return float(e[0]), g[0].cpu().numpy() @ self.A


def get_state(*_, **__):
    raise RuntimeError("Dense state extraction is not supported by the MPS engine")
