"""Plain partition warm start on the engine: graph communities, local VQEs, then
one global refinement.

Restates ``IndependentSubspaceVQE`` (test/sources/independent-vqe/Qiskit_VQE/
independent_vqe.py) for the MPS engine:

* the weighted qubit-coupling graph (:62-68; every pair of qubits in a term's
  support gains |c|) and ``_partition`` (:140-158): networkx Louvain
  communities per connected component with the strategy's seed, then
  Kernighan-Lin bisection of any community wider than ``max_block_qubits``;
* local models (:73-104): terms inside one block, constant terms to block 0,
  width max(2, |block|), parameters mapped by (layer, qubit, gate);
* ``_minimize_model`` (:176-245) for every block and for the global problem:
  L-BFGS-B (ftol 1e-12, gtol 1e-8) or COBYLA (tol 1e-8), cost cache, best
  tracking, and the callback's early stop once an accepted step improves the
  energy by less than ``energy_tol``;
* ``_run_vqe`` (:257-323): seeded uniform start, local solves, assembled warm
  start, one global refinement.

What changes is how the work reaches the GPU. The local solves run
concurrently -- one optimizer thread per block -- and every round of their
energy requests is ONE partition-set call (all blocks, all requested points,
in one batch) instead of one observe() per point and block. The local
gradient is the reference's parameter-shift rule (:206-214), its 2P shifted
points requested together with the centre point. The global gradient is the
engine's adjoint (``Engine.energy_grad``), equal to the parameter-shift
gradient of these rotation circuits up to rounding, at the cost of a few
energy evaluations instead of 2P of them.
"""
from __future__ import annotations

import threading
import time
from itertools import combinations

import numpy as np
from . import _lib, optimize
from ._lib import EngineError


def simplify(words, coeffs):
    """Merge identical words (coefficients summed, first occurrence kept) and drop
    exact zeros, as ``SparsePauliOp.simplify(atol=0, rtol=0)`` (:53)."""
    pos, w_out, c_out = {}, [], []
    for w, c in zip(words, coeffs):
        i = pos.get(w)
        if i is None:
            pos[w] = len(w_out)
            w_out.append(w)
            c_out.append(float(c))
        else:
            c_out[i] += float(c)
    keep = [i for i, c in enumerate(c_out) if c != 0.0]
    return [w_out[i] for i in keep], np.array([c_out[i] for i in keep], dtype=float)


def pairs_for_pattern(n, pattern):
    """CX pairs of one entangling layer (efficientsu2.py:23-43)."""
    if pattern == "linear":
        return [(i, i + 1) for i in range(n - 1)]
    if pattern == "reverse_linear":
        return [(i, i + 1) for i in range(n - 2, -1, -1)]
    raise ValueError("Expected linear or reverse_linear")


def ansatz_ops(n_active, reps, gates, pattern):
    """Op list of the nearest-neighbour SU(2) ansatz over qubits 0..n_active-1
    (``_build_kernel``, :160-174): per layer every qubit's rotations in
    (qubit, gate) order, then the CX chain (none for a single qubit)."""
    ops, index = [], 0
    for layer in range(reps + 1):
        for q in range(n_active):
            for g in gates:
                ops.append((g, q, index))
                index += 1
        if layer < reps and n_active > 1:
            ops.extend(("cx", a, b) for a, b in pairs_for_pattern(n_active, pattern))
    return ops, index


class _RoundBatcher:
    """Collects the energy requests of concurrently running block optimizers and
    answers each round with one partition-set call (runs on the calling thread)."""

    def __init__(self, engine, pset, blocks_params):
        self.engine = engine
        self.pset = pset
        self.P = blocks_params
        self.cv = threading.Condition()
        self.pending = {}
        self.results = {}
        self.active = set(range(pset.K))
        self.calls = 0
        self.points = 0

    def request(self, k, X):
        with self.cv:
            self.pending[k] = np.asarray(X, dtype=float).reshape(-1, self.P[k])
            self.cv.notify_all()
            while k not in self.results:
                self.cv.wait()
            out = self.results.pop(k)
        if isinstance(out, BaseException):
            raise out
        return out

    def finish(self, k):
        with self.cv:
            self.active.discard(k)
            self.cv.notify_all()

    def serve(self):
        import torch
        while True:
            with self.cv:
                while self.active and not (self.pending and set(self.pending) >= self.active):
                    self.cv.wait()
                if not self.active:
                    return
                batch, self.pending = self.pending, {}
            copies = max(len(X) for X in batch.values())
            theta = np.zeros((self.pset.K * copies, self.pset.P_max))
            for k, X in batch.items():
                rows = slice(k * copies, k * copies + len(X))
                theta[rows, :self.P[k]] = X
            try:
                e = self.engine.partition_energy(self.pset, torch.from_numpy(theta).to(self.engine.device),
                                                 copies=copies).cpu().numpy()
                answers = {k: e[k * copies:k * copies + len(X)].copy() for k, X in batch.items()}
            except BaseException as exc:   # hand the failure to every waiting optimizer
                answers = {k: exc for k in batch}
            self.calls += 1
            self.points += sum(len(X) for X in batch.values())
            with self.cv:
                self.results.update(answers)
                self.cv.notify_all()


def minimize_model(params, maxiter, constant, energies, value_grad, *, energy_tol=1.0,
                   use_gradient_optimizer=True, line_search="scipy"):
    """One model's optimisation (independent_vqe.py:176-245) through the drivers
    of :mod:`vqemps.optimize`: L-BFGS-B (ftol 1e-12, gtol 1e-8) or COBYLA (tol
    1e-8), both stopping once an accepted iterate improves the energy by less
    than ``energy_tol``.

    ``energies(X)`` -> energies of the rows of X; ``value_grad(x)`` -> (E, dE/dx),
    or None to use the parameter-shift rule through ``energies`` (the 2P shifted
    points and the centre in one call). ``line_search="batched"`` evaluates the
    L-BFGS step lengths several per call (:func:`vqemps.optimize.lbfgs_batched`)."""
    params = np.asarray(params, dtype=float).copy()
    history = []
    accepted = [0]

    def evaluate_with_gradient(x):
        x = np.asarray(x, dtype=float)
        if value_grad is not None:
            e, g = value_grad(x)
        else:
            P = x.size
            shifted = np.repeat(x[None, :], 2 * P + 1, axis=0)
            idx = np.arange(P)
            shifted[1 + idx, idx] += np.pi / 2
            shifted[1 + P + idx, idx] -= np.pi / 2
            v = energies(shifted)
            e, g = v[0], (v[1:P + 1] - v[P + 1:]) / 2
        history.append(float(e))
        return float(e), np.asarray(g, dtype=float)

    def evaluate_batch(X):
        out = [evaluate_with_gradient(x) for x in np.atleast_2d(X)]
        return np.array([o[0] for o in out]), np.array([o[1] for o in out])

    def energy_only(x):
        e = float(energies(np.asarray(x, dtype=float)[None, :])[0])
        history.append(e)
        return e

    def count(_x):
        accepted[0] += 1

    started = time.perf_counter()
    if maxiter and not constant:
        if use_gradient_optimizer:
            res = optimize.lbfgs_minimize(evaluate_with_gradient, params, maxiter=maxiter, ftol=1e-12, gtol=1e-8,
                                          immediate_energy_tol=None, accepted_energy_tol=energy_tol, callback=count,
                                          line_search=line_search, value_grad_batch=evaluate_batch)
            energy, best_x = float(res.get("best_energy", res.fun)), np.asarray(res.get("best_x", res.x))
        else:
            res = optimize.cobyla_minimize(energy_only, params, maxiter, tol=1e-8, accepted_energy_tol=energy_tol,
                                           callback=count)
            energy, best_x = float(res.fun), np.asarray(res.x)
        reason = str(res.message)
    else:
        energy = evaluate_with_gradient(params)[0] if use_gradient_optimizer else energy_only(params)
        best_x = params.copy()
        reason = "constant_local_objective" if constant else "iteration_limit"
    return dict(energy=float(energy), params=best_x, accepted_iterations=accepted[0], stop_reason=reason,
                duration_s=time.perf_counter() - started, history=history)


class PartitionPlan:
    """Host-only part of the strategy: simplified Hamiltonian, coupling graph,
    blocks and local models (no GPU needed).

    ``words`` are qubit-indexed Pauli strings (word[q] acts on qubit q).
    """

    def __init__(self, n, words, coeffs, *, reps=4, su2_gates=("ry",), entanglement="linear",
                 max_block_qubits=12, blocks=None, seed=0):
        import networkx as nx
        if entanglement not in ("linear", "reverse_linear"):
            raise ValueError("Expected linear or reverse_linear")
        if any(g not in ("rx", "ry", "rz") for g in su2_gates):
            raise ValueError("Parameter-shift requires rx, ry, or rz rotations")
        if max_block_qubits is not None and max_block_qubits < 1:
            raise ValueError("max_block_qubits must be positive or None")
        self.n = n
        self.reps = reps
        self.gates = tuple(su2_gates)
        self.entanglement = entanglement
        self.max_block_qubits = max_block_qubits
        self.seed = seed
        self.words, self.coeffs = simplify(list(words), np.asarray(coeffs, dtype=float))
        for w in self.words:
            if len(w) != n:
                raise EngineError(_lib.INVALID, "Hamiltonian/register width mismatch")
        self.graph = nx.Graph()
        self.graph.add_nodes_from(range(n))
        for w, c in zip(self.words, self.coeffs):
            support = [q for q, p in enumerate(w) if p != "I"]
            for a, b in combinations(support, 2):
                if abs(c):
                    weight = self.graph.get_edge_data(a, b, {}).get("weight", 0.0)
                    self.graph.add_edge(a, b, weight=weight + float(abs(c)))
        self.blocks = self._partition() if blocks is None else [sorted(b) for b in blocks]
        flat = sorted(q for b in self.blocks for q in b)
        if any(not b for b in self.blocks) or flat != list(range(n)):
            raise ValueError("Blocks must cover each qubit exactly once")
        self._build_local_models()
        self.global_ops, self.num_params = ansatz_ops(n, reps, self.gates, entanglement)

    # -- partition (independent_vqe.py:140-158) ------------------------------
    def _partition(self):
        import networkx as nx
        communities = []
        for component in nx.connected_components(self.graph):
            sub = self.graph.subgraph(component)
            if sub.number_of_edges():
                communities.extend(nx.community.louvain_communities(sub, weight="weight", seed=self.seed))
            else:
                communities.extend({q} for q in component)
        pending, result = list(communities), []
        while pending:
            block = pending.pop()
            if self.max_block_qubits is None or len(block) <= self.max_block_qubits:
                result.append(sorted(block))
            else:
                left, right = nx.community.kernighan_lin_bisection(
                    self.graph.subgraph(sorted(block)), weight="weight", seed=self.seed)
                pending.extend((left, right))
        return sorted(result, key=lambda b: b[0])

    # -- local models (independent_vqe.py:73-104) ----------------------------
    def _build_local_models(self):
        owner = {q: i for i, b in enumerate(self.blocks) for q in b}
        local = [[] for _ in self.blocks]
        self.cross_terms = []
        for w, c in zip(self.words, self.coeffs):
            support = [q for q, p in enumerate(w) if p != "I"]
            owners = {owner[q] for q in support}
            if len(owners) > 1:
                self.cross_terms.append((w, float(c)))
                continue
            i = next(iter(owners)) if owners else 0
            block = self.blocks[i]
            chars = [w[q] for q in block] + ["I"] * (max(2, len(block)) - len(block))
            local[i].append(("".join(chars), float(c)))
        G = len(self.gates)
        self.local_models = []
        for i, block in enumerate(self.blocks):
            width = max(2, len(block))
            terms = local[i] or [("I" * width, 0.0)]
            ops, count = ansatz_ops(len(block), self.reps, self.gates, self.entanglement)
            self.local_models.append(dict(
                qubits=list(block), width=width, terms=terms, ops=ops, count=count,
                constant=all(set(t) <= {"I"} for t, _ in terms),
                parameter_indices=np.array([(layer * self.n + q) * G + g for layer in range(self.reps + 1)
                                            for q in block for g in range(G)], dtype=np.int64)))

class GlobalProblem:
    """The full-width objective on the engine: the nearest-neighbour ansatz over
    all qubits and the whole Hamiltonian (``_build_kernel([range(n)], ...)``,
    independent_vqe.py:106-110), with the energy, the adjoint value/gradient and
    the global refinement."""

    def __init__(self, engine, n, words, coeffs, *, reps=4, su2_gates=("ry",), entanglement="linear",
                 energy_tol=1.0, use_gradient_optimizer=True):
        self.engine = engine
        self.n = n
        self.energy_tol = energy_tol
        self.use_gradient_optimizer = use_gradient_optimizer
        self.ops, self.num_params = ansatz_ops(n, reps, tuple(su2_gates), entanglement)
        width = max(2, n)
        engine.set_circuit(width, self.ops, site_order="msb")
        words = [w + "I" * (width - n) for w in words] or ["I" * width]
        self.ham = engine.set_hamiltonian(words, coeffs if len(coeffs) else [0.0])

    def energy(self, theta):
        import torch
        t = torch.as_tensor(np.atleast_2d(theta), dtype=torch.float64, device=self.engine.device)
        return self.engine.energy(self.ham, t).cpu().numpy()

    def value_grad(self, theta):
        import torch
        t = torch.as_tensor(np.atleast_2d(theta), dtype=torch.float64, device=self.engine.device)
        e, g = self.engine.energy_grad(self.ham, t)
        return float(e[0]), g[0].cpu().numpy()

    def refine(self, theta, maxiter):
        return minimize_model(theta, maxiter, False, self.energy,
                              self.value_grad if self.use_gradient_optimizer else None,
                              energy_tol=self.energy_tol, use_gradient_optimizer=self.use_gradient_optimizer)


class IndependentPartitionVQE:
    """Partition warm start + global refinement of one Hamiltonian on one engine.

    Defaults follow IndependentSubspaceVQE's (max_block_qubits 12, energy_tol
    1.0, linear chain, block_maxiter 30, global_maxiter 10, reps 4, seed 0);
    the rotation set defaults to RY only, the synthetic workloads' ansatz.
    """

    def __init__(self, engine, n, words, coeffs, *, reps=4, su2_gates=("ry",), entanglement="linear",
                 max_block_qubits=12, blocks=None, energy_tol=1.0, block_maxiter=30, global_maxiter=10,
                 use_gradient_optimizer=True, global_refinement=True, seed=0):
        if not np.isfinite(energy_tol) or energy_tol <= 0:
            raise ValueError("energy_tol must be positive")
        self.plan = PartitionPlan(n, words, coeffs, reps=reps, su2_gates=su2_gates, entanglement=entanglement,
                                  max_block_qubits=max_block_qubits, blocks=blocks, seed=seed)
        self.engine = engine
        self.n = n
        self.energy_tol = energy_tol
        self.block_maxiter = block_maxiter
        self.global_maxiter = global_maxiter
        self.use_gradient_optimizer = use_gradient_optimizer
        self.global_refinement = global_refinement
        self.seed = seed
        self.blocks = self.plan.blocks
        self.local_models = self.plan.local_models
        self.num_params = self.plan.num_params
        self.problem = GlobalProblem(engine, n, self.plan.words, self.plan.coeffs, reps=reps, su2_gates=su2_gates,
                                     entanglement=entanglement, energy_tol=energy_tol,
                                     use_gradient_optimizer=use_gradient_optimizer)

    # -- local phase: all blocks at once ---------------------------------------
    def solve_locals(self, theta):
        """Run every block's local optimisation concurrently; one partition-set
        call per round of requests. Returns the per-block results."""
        eng = self.engine
        pset = eng.set_partitions([(m["width"], m["ops"], [t for t, _ in m["terms"]], [c for _, c in m["terms"]])
                                   for m in self.local_models], site_order="msb")
        batcher = _RoundBatcher(eng, pset, [m["count"] for m in self.local_models])
        results = [None] * len(self.local_models)
        errors = []

        def work(k):
            try:
                m = self.local_models[k]
                results[k] = minimize_model(theta[m["parameter_indices"]], self.block_maxiter, m["constant"],
                                            lambda X: batcher.request(k, X), None, energy_tol=self.energy_tol,
                                            use_gradient_optimizer=self.use_gradient_optimizer)
            except BaseException as exc:
                errors.append(exc)
            finally:
                batcher.finish(k)

        threads = [threading.Thread(target=work, args=(k,), daemon=True) for k in range(len(self.local_models))]
        for t in threads:
            t.start()
        batcher.serve()
        for t in threads:
            t.join()
        eng.free_partitions(pset)
        if errors:
            raise errors[0]
        self.local_calls, self.local_points = batcher.calls, batcher.points
        return results

    # -- global objective ------------------------------------------------------
    def energy(self, theta):
        return self.problem.energy(theta)

    def value_grad(self, theta):
        return self.problem.value_grad(theta)

    def refine(self, theta, maxiter=None):
        """Global refinement from ``theta`` (the reference's global _minimize_model)."""
        return self.problem.refine(theta, self.global_maxiter if maxiter is None else maxiter)

    def initial_theta(self):
        return np.random.default_rng(self.seed).uniform(-np.pi, np.pi, self.num_params)

    def run(self, init_params=None):
        """The whole plain method: local solves, warm start, global refinement."""
        t0 = time.perf_counter()
        theta = self.initial_theta() if init_params is None else np.asarray(init_params, dtype=float).copy()
        if theta.shape != (self.num_params,) or not np.all(np.isfinite(theta)):
            raise ValueError(f"Expected {self.num_params} finite initial parameters")
        local = self.solve_locals(theta)
        for m, r in zip(self.local_models, local):
            theta[m["parameter_indices"]] = r["params"]
        t1 = time.perf_counter()
        warm_energy = float(self.energy(theta)[0])
        out = dict(blocks=self.blocks, local_results=local, warm_start_params=theta.copy(),
                   warm_start_energy=warm_energy, local_s=t1 - t0, local_calls=self.local_calls,
                   local_points=self.local_points, crossing_term_count=len(self.plan.cross_terms))
        best_e, best_x = warm_energy, theta.copy()
        if self.global_refinement and self.global_maxiter > 0:
            g = self.refine(theta)
            out["global_result"] = {k: v for k, v in g.items() if k != "params"}
            if g["energy"] < best_e:
                best_e, best_x = g["energy"], g["params"]
        out.update(best_energy=best_e, best_params=best_x, total_s=time.perf_counter() - t0)
        return out
