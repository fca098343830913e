"""Test infrastructure (the oracle): sequential restatements of the reference's
optimizer and partition-strategy logic, one scalar objective call at a time.

Only tests may import this module. Functions cite the reference lines they
restate.
"""
from __future__ import annotations

from itertools import combinations

import numpy as np


def spsa_sequential(fun, x0, maxiter, perturbation=0.2, learning_rate=None, alpha=0.602, gamma=0.101,
                    stability=0.0, calibration_pairs=5, target_update=2 * np.pi / 10, seed=0,
                    immediate_energy_tol=1.0):
    """test/tools/spsa_optimizer.py:66-187 without journaling/logging: returns
    (best_x, best_f, nit, nfev, trajectory of accepted x)."""
    x = np.asarray(x0, dtype=float).copy()
    rng = np.random.default_rng(seed)
    nfev = 0

    def ev(p):
        nonlocal nfev
        nfev += 1
        return float(fun(p))

    def pgrad(xx, c):                         # perturbation_gradient :58-63
        delta = rng.choice(np.array([-1., 1.]), size=xx.size)
        plus = ev(xx + c * delta)
        minus = ev(xx - c * delta)
        return ((plus - minus) / (2 * c)) * delta

    fx = ev(x)
    best_x, best_f = x.copy(), fx
    c, a = perturbation, learning_rate
    if a is None:                             # :129-138
        mags = [float(np.mean(np.abs(pgrad(x, c)))) for _ in range(calibration_pairs)]
        m = float(np.mean(mags))
        a = target_update * (stability + 1) ** alpha / m if m > 1e-12 else 1.0
    traj = []
    nit = 0
    for k in range(1, maxiter + 1):           # :142-176
        prev = fx
        ak = a / (k + stability) ** alpha
        ck = c / k ** gamma
        g = pgrad(x, ck)
        cand = x - ak * g
        fx = ev(cand)
        x = cand
        nit = k
        traj.append(x.copy())
        if fx < best_f:
            best_x, best_f = x.copy(), fx
        if immediate_energy_tol is not None and abs(fx - prev) < immediate_energy_tol:
            break
    return best_x, best_f, nit, nfev, traj


def simplify_terms(words, coeffs):
    """SparsePauliOp.simplify(atol=0, rtol=0) as the strategy uses it
    (independent_vqe.py:53): identical words merge by summing coefficients in
    order of first occurrence; exact zeros are dropped."""
    index, out_w, out_c = {}, [], []
    for w, c in zip(words, coeffs):
        if w in index:
            out_c[index[w]] += float(c)
        else:
            index[w] = len(out_w)
            out_w.append(w)
            out_c.append(float(c))
    keep = [i for i, c in enumerate(out_c) if c != 0.0]
    return [out_w[i] for i in keep], [out_c[i] for i in keep]


def coupling_edges(words, coeffs):
    """Weighted coupling graph of independent_vqe.py:62-68 as {(a, b): weight}:
    every pair of qubits in a term's support gains |c| (words indexed by qubit)."""
    edges = {}
    for w, c in zip(words, coeffs):
        support = [q for q, p in enumerate(w) if p != "I"]
        for a, b in combinations(support, 2):
            if abs(c):
                edges[(a, b)] = edges.get((a, b), 0.0) + float(abs(c))
    return edges


def local_problems(n, blocks, words, coeffs, reps, gates=("ry",)):
    """Local terms, widths and parameter maps of independent_vqe.py:73-104:
    returns (local models, cross terms). A local word is indexed by the block's
    local qubit (word[i] acts on block[i]), padded with I to max(2, len(block));
    constant words go to block 0; parameter_indices follow (layer, qubit, gate)."""
    owner = {q: i for i, b in enumerate(blocks) for q in b}
    local = [[] for _ in blocks]
    cross = []
    for w, c in zip(words, coeffs):
        if c == 0:
            continue
        support = [q for q, p in enumerate(w) if p != "I"]
        owners = {owner[q] for q in support}
        if len(owners) > 1:
            cross.append((w, float(c)))
            continue
        i = next(iter(owners)) if owners else 0
        block = blocks[i]
        chars = [w[q] for q in block]
        chars += ["I"] * (max(2, len(block)) - len(block))
        local[i].append(("".join(chars), float(c)))
    G = len(gates)
    models = []
    for i, block in enumerate(blocks):
        width = max(2, len(block))
        terms = local[i] or [("I" * width, 0.0)]
        models.append(dict(qubits=list(block), width=width, terms=terms,
                           constant=all(set(t) <= {"I"} for t, _ in terms),
                           parameter_indices=[(layer * n + q) * G + g for layer in range(reps + 1)
                                              for q in block for g in range(G)]))
    return models, cross
