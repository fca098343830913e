"""CPU oracle for the MPS VQE hot path -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it.
The CUDA engine in ``graph-vqe_b200/`` never routes through it.

It restates, in numpy complex128, the reference algorithms of hp-cyber/Graph-VQE
that lie on the hot path (paths relative to the reference project root):

* circuit specs ........ test/tools/reverse_mps.py:12-25 (``register``),
                         test/sources/independent-vqe/Qiskit_VQE/efficientsu2.py:23-43
* exact bond-doubling MPS  test/tools/reverse_mps.py:39-57 (``ReverseMPS.sites``)
* prefix-shared energy . test/tools/reverse_mps.py:59-82 (``energy_chunk``) and
                         test/backend/source/sharded_mps.cuh:614-687,
                         test/backend/source/analytic_batch.cuh:4-36
* SVD gate evolution ... test/backend/source/sharded_mps.cuh:465-572 (apply1q/apply2q/
                         applyTwoQubit), dist_svd.cuh:194-283 (zero-cutoff direct SVD,
                         rank guard, factor packing)
* perfect sampling ..... test/backend/source/sharded_mps.cuh:61-188,814-877,986-1035
* diagonal shot sums ... test/backend/source/sharded_mps.cuh:193-214,906-935
* seeds ................ test/backend/source/simulator_mps_dist.cu:214,586-608

Parity is pinned against golden vectors produced by the reference's own
``ReverseMPS`` (tests/golden/make_golden.py) and against the known-answer tests of
test/setup_local_cudaq.sh:3019-3100 and test/tests/test_reverse_mps.py.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# ---------------------------------------------------------------------------
# Circuit specifications
# ---------------------------------------------------------------------------

ROTATIONS = ("rx", "ry", "rz")
FIXED_1Q = ("h", "x", "y", "z", "s", "sdg")
INITIAL_VECTORS = {
    None: (1.0, 0.0), "0": (1.0, 0.0), "1": (0.0, 1.0),
    "+": (2 ** -0.5, 2 ** -0.5), "-": (2 ** -0.5, -(2 ** -0.5)),
}


def pairs_for_pattern(n: int, layer: int, pattern: str):
    """CX pairs of one entangling layer (efficientsu2.py:23-43).

    ``linear`` gives (i, i+1) for i = 0..n-2; ``reverse_linear`` gives the same
    pairs for i = n-2..0. Other patterns of the reference are outside the hot path.
    """
    del layer
    p = pattern.lower()
    if p == "linear":
        return [(i, i + 1) for i in range(n - 1)]
    if p == "reverse_linear":
        return [(i, i + 1) for i in range(n - 2, -1, -1)]
    raise ValueError(f"unsupported entanglement pattern: {pattern}")


def hardware_efficient_spec(n: int, reps: int, gates=("ry",), pattern="linear",
                            initial=None):
    """Op list of the hardware-efficient ansatz in ``register`` form.

    Parameter order is (layer, qubit, gate) as in independent_vqe.py:108-110 and
    reverse_mps.py:16-24; each layer's rotations come before its CX chain and a
    final rotation layer closes the circuit.
    ops: ``(gate, qubit, param_index)`` for rotations, ``('cx', control, target)``.
    """
    ops = []
    index = 0
    for layer in range(reps + 1):
        for q in range(n):
            for g in gates:
                ops.append((g.lower(), q, index))
                index += 1
        if layer < reps:
            ops.extend(("cx", c, t) for c, t in pairs_for_pattern(n, layer, pattern))
    return dict(n=n, ops=ops, initial=initial, count=index)


def configure_full_bond(num_qubits: int, stages=None) -> int:
    """Exact bond cap of nearest-neighbour circuits (mps_config.py:8-43), without
    the environment side effects: 2**min(reps, n//2) for linear/reverse_linear,
    2**min(ceil(reps/2), n//2) for pairwise, 2**(n//2) otherwise, saturating at
    2**31 - 1."""
    if num_qubits < 2:
        raise ValueError("at least two qubits are required")
    exponents = []
    for stage in stages or [{"entanglement": None}]:
        exponent = num_qubits // 2
        pattern = stage.get("entanglement")
        reps = stage.get("reps")
        if isinstance(pattern, str) and reps is not None:
            reps = int(reps)
            if reps < 0:
                raise ValueError("reps must be nonnegative")
            if pattern.lower() in ("linear", "reverse_linear"):
                exponent = min(exponent, reps)
            elif pattern.lower() == "pairwise":
                exponent = min(exponent, (reps + 1) // 2)
        exponents.append(exponent)
    exponent = max(exponents)
    return (1 << exponent) if exponent < 31 else 2 ** 31 - 1


def rotation(gate: str, angle: float) -> np.ndarray:
    """CUDA-Q rotation matrices as used in reverse_mps.py:52-56."""
    c, s = math.cos(angle / 2), math.sin(angle / 2)
    if gate == "ry":
        return np.array([[c, -s], [s, c]], dtype=complex)
    if gate == "rx":
        return np.array([[c, -1j * s], [-1j * s, c]], dtype=complex)
    if gate == "rz":
        return np.diag([np.exp(-0.5j * angle), np.exp(0.5j * angle)])
    raise ValueError(gate)


def rotation_derivative(gate: str, angle: float) -> np.ndarray:
    """d/d(angle) of ``rotation``."""
    c, s = math.cos(angle / 2), math.sin(angle / 2)
    if gate == "ry":
        return 0.5 * np.array([[-s, -c], [c, -s]], dtype=complex)
    if gate == "rx":
        return 0.5 * np.array([[-s, -1j * c], [-1j * c, -s]], dtype=complex)
    if gate == "rz":
        return np.diag([-0.5j * np.exp(-0.5j * angle), 0.5j * np.exp(0.5j * angle)])
    raise ValueError(gate)


FIXED_MATRICES = {
    "h": np.array([[1, 1], [1, -1]], dtype=complex) / math.sqrt(2),
    "x": np.array([[0, 1], [1, 0]], dtype=complex),
    "y": np.array([[0, -1j], [1j, 0]], dtype=complex),
    "z": np.array([[1, 0], [0, -1]], dtype=complex),
    "s": np.array([[1, 0], [0, 1j]], dtype=complex),
    "sdg": np.array([[1, 0], [0, -1j]], dtype=complex),
}


def op_matrix(op, x):
    gate = op[0]
    if gate in ROTATIONS:
        return rotation(gate, float(x[op[2]]))
    return FIXED_MATRICES[gate]


# ---------------------------------------------------------------------------
# Exact bond-doubling MPS (reverse_mps.py:39-57) and its energy (:59-82)
# ---------------------------------------------------------------------------

def bond_doubling_sites(spec, x):
    """Exact MPS without SVD: a CX doubles the bond between its two sites.

    Site tensors are (left, physical, right), site index = qubit index.
    ``left = A (x) I`` and ``right = stack(B, flip(B))`` (reverse_mps.py:45-50);
    a CX whose control is the right-hand site mirrors that construction
    (reverse_mps.py:162-168).
    """
    n = spec["n"]
    vec = np.array(INITIAL_VECTORS[spec.get("initial")], dtype=complex)
    sites = [vec.reshape(1, 2, 1).copy() for _ in range(n)]
    for op in spec["ops"]:
        if op[0] == "cx":
            c, t = op[1], op[2]
            lo, hi = min(c, t), max(c, t)
            if hi != lo + 1:
                raise ValueError("bond doubling needs adjacent CX pairs")
            a, b = sites[lo], sites[hi]
            if c == lo:
                left = np.einsum("aib,is->aibs", a, np.eye(2)).reshape(a.shape[0], 2, a.shape[2] * 2)
                right = np.stack((b, b[:, ::-1, :]), axis=1).reshape(b.shape[0] * 2, 2, b.shape[2])
            else:
                left = np.stack((a, a[:, ::-1, :]), axis=-1).reshape(a.shape[0], 2, a.shape[2] * 2)
                right = np.einsum("aib,is->asib", b, np.eye(2)).reshape(b.shape[0] * 2, 2, b.shape[2])
            sites[lo], sites[hi] = left, right
        else:
            m = op_matrix(op, x)
            q = op[1]
            sites[q] = np.einsum("ij,ajb->aib", m, sites[q])
    return sites


PAULI = {
    "I": np.eye(2, dtype=complex),
    "X": np.array([[0, 1], [1, 0]], dtype=complex),
    "Y": np.array([[0, -1j], [1j, 0]], dtype=complex),
    "Z": np.array([[1, 0], [0, -1]], dtype=complex),
}


def transfer(env, a, p):
    """E'[b,c] = sum conj(A[a,i,b]) P[i,i'] E[a,a'] A[a',i',c] (analytic_batch.cuh:4-31)."""
    s = np.einsum("xab,bic->xaic", env, a)            # E * A
    s = np.einsum("ij,xajc->xaic", PAULI[p], s)        # Pauli on the ket side
    return np.einsum("aib,xaic->xbc", a.conj(), s)


def prefix_levels(words, n):
    """Prefix trie over ``words`` in the given order (reverse_mps.py:62-70).

    Returns, per site q, (parents, paulis) of the distinct (parent, pauli) nodes
    and the leaf node of every word after the last site.
    """
    previous = [0] * len(words)
    levels = []
    for q in range(n):
        nodes = {}
        parents, paulis, current = [], [], []
        for prev, word in zip(previous, words):
            key = (prev, word[q])
            if key not in nodes:
                nodes[key] = len(nodes)
                parents.append(prev)
                paulis.append(word[q])
            current.append(nodes[key])
        levels.append((parents, paulis))
        previous = current
    return levels, previous


def expect_words(sites, words):
    """<psi|P|psi> of each word by a prefix-shared left sweep (energy_chunk)."""
    if not words:
        return np.zeros(0, dtype=complex)
    n = len(sites)
    levels, leaves = prefix_levels(words, n)
    env = np.ones((1, 1, 1), dtype=complex)
    for q, (parents, paulis) in enumerate(levels):
        incoming = env[np.asarray(parents)]
        out = np.empty((len(parents), sites[q].shape[2], sites[q].shape[2]), dtype=complex)
        for p in "IXYZ":
            idx = [j for j, c in enumerate(paulis) if c == p]
            if idx:
                out[idx] = transfer(incoming[idx], sites[q], p)
        env = out
    return env[np.asarray(leaves), 0, 0]


def reverse_energy(spec, words, coeffs, x, chunk=128):
    """Energy of ReverseMPS in chunks of ``chunk`` terms (reverse_mps.py:84-99)."""
    sites = bond_doubling_sites(spec, x)
    total = 0.0
    for start in range(0, len(words), chunk):
        vals = expect_words(sites, words[start:start + chunk]).real
        total += float(np.dot(vals, coeffs[start:start + chunk]))
    return total


def reverse_value_gradient(spec, words, coeffs, x):
    """Energy and d(energy)/d(theta) by a hand-written adjoint of the exact MPS.

    Same quantity as ``ReverseMPS.value_gradient`` (reverse_mps.py:84-99), which
    gets it from torch autograd. Forward: bond-doubling sites, full left sweep per
    prefix node. Backward: the adjoint transfer E_bar = sum conj(P) A_i Ebar' A_i'^H
    down the trie, site cotangents A_bar_i += 2 sum_i' P[i,i'] E A_i' Ebar',
    then back through the gate list (rotations and CX doublings).
    """
    n = spec["n"]
    ops = spec["ops"]
    coeffs = np.asarray(coeffs, dtype=float)
    # forward through the gates, recording inputs of rotations
    vec = np.array(INITIAL_VECTORS[spec.get("initial")], dtype=complex)
    sites = [vec.reshape(1, 2, 1).copy() for _ in range(n)]
    tape = []
    for op in ops:
        if op[0] == "cx":
            c, t = op[1], op[2]
            lo, hi = min(c, t), max(c, t)
            a, b = sites[lo], sites[hi]
            tape.append((a.shape, b.shape))
            if c == lo:
                left = np.einsum("aib,is->aibs", a, np.eye(2)).reshape(a.shape[0], 2, a.shape[2] * 2)
                right = np.stack((b, b[:, ::-1, :]), axis=1).reshape(b.shape[0] * 2, 2, b.shape[2])
            else:
                left = np.stack((a, a[:, ::-1, :]), axis=-1).reshape(a.shape[0], 2, a.shape[2] * 2)
                right = np.einsum("aib,is->asib", b, np.eye(2)).reshape(b.shape[0] * 2, 2, b.shape[2])
            sites[lo], sites[hi] = left, right
        else:
            tape.append(sites[op[1]])
            sites[op[1]] = np.einsum("ij,ajb->aib", op_matrix(op, x), sites[op[1]])
    # trie forward keeping every level
    levels, leaves = prefix_levels(list(words), n)
    envs = [np.ones((1, 1, 1), dtype=complex)]
    for q, (parents, paulis) in enumerate(levels):
        incoming = envs[-1][np.asarray(parents)]
        out = np.empty((len(parents), sites[q].shape[2], sites[q].shape[2]), dtype=complex)
        for p in "IXYZ":
            idx = [j for j, c in enumerate(paulis) if c == p]
            if idx:
                out[idx] = transfer(incoming[idx], sites[q], p)
        envs.append(out)
    values = envs[-1][np.asarray(leaves), 0, 0].real
    energy = float(np.dot(values, coeffs))
    # backward down the trie
    bar = np.zeros_like(envs[-1])
    np.add.at(bar[:, 0, 0], np.asarray(leaves), coeffs.astype(complex))
    site_bar = [np.zeros_like(s) for s in sites]
    for q in range(n - 1, -1, -1):
        parents, paulis = levels[q]
        a = sites[q]
        parent_env = envs[q][np.asarray(parents)]
        parent_bar = np.zeros_like(envs[q])
        for p in "IXYZ":
            idx = [j for j, c in enumerate(paulis) if c == p]
            if not idx:
                continue
            pm = PAULI[p]
            eb = bar[idx]                                   # child cotangents
            e = parent_env[idx]
            # S'[x,a,i,c] = sum_i' P[i,i'] (E A_i')[x,a,c]
            s = np.einsum("xab,bjc->xajc", e, a)
            s = np.einsum("ij,xajc->xaic", pm, s)
            site_bar[q] += 2.0 * np.einsum("xaic,xcd->aid", s, eb)
            # E_bar = sum conj(P[i,i']) A_i Ebar' A_i'^H
            t = np.einsum("aib,xbc->xaic", a, eb)
            t = np.einsum("ij,xaic->xajc", pm.conj(), t)
            contrib = np.einsum("xajc,djc->xad", t, a.conj())
            np.add.at(parent_bar, np.asarray(parents)[idx], contrib)
        bar = parent_bar
    # backward through the gates
    grad = np.zeros(len(x))
    for op, saved in zip(reversed(ops), reversed(tape)):
        if op[0] == "cx":
            c, t = op[1], op[2]
            lo, hi = min(c, t), max(c, t)
            (ash, bsh) = saved
            lb, rb = site_bar[lo], site_bar[hi]
            lb4 = lb.reshape(ash[0], 2, ash[2], 2)
            rb4 = rb.reshape(bsh[0], 2, 2, bsh[2])
            if c == lo:
                abar = np.stack([lb4[:, i, :, i] for i in range(2)], axis=1)
                bbar = rb4[:, 0] + rb4[:, 1, ::-1]
            else:
                abar = lb4[..., 0] + lb4[:, ::-1, :, 1]
                bbar = np.stack([rb4[:, i, i, :] for i in range(2)], axis=1)
            site_bar[lo], site_bar[hi] = abar, bbar
        else:
            q = op[1]
            a_old = saved
            nbar = site_bar[q]
            if op[0] in ROTATIONS:
                dm = rotation_derivative(op[0], float(x[op[2]]))
                grad[op[2]] += float(np.real(np.vdot(nbar, np.einsum("ij,ajb->aib", dm, a_old))))
            m = op_matrix(op, x)
            site_bar[q] = np.einsum("ij,aib->ajb", m.conj(), nbar)
    return energy, grad


# ---------------------------------------------------------------------------
# SVD gate evolution of the backend (sharded_mps.cuh + dist_svd.cuh)
# ---------------------------------------------------------------------------

EPS = 2.2204460492503131e-16


class InsufficientBond(RuntimeError):
    """dist_svd.cuh:277-279 -- a resolved singular value would be discarded."""


class NonfiniteSvd(RuntimeError):
    """dist_svd.cuh:280-281 -- the SVD failed or produced nonfinite values."""


def select_rank(singular, max_bond, abs_cut=0.0, rel_cut=0.0):
    """``selectDirectSvdRank`` (dist_svd.cuh:194-212): -1 nonfinite, -2 cap too small."""
    count = len(singular)
    threshold = max(abs_cut, rel_cut * singular[0])
    selected = 0
    for v in singular:
        if not np.isfinite(v) or v < 0.0:
            return -1
        if (abs_cut == 0.0 and rel_cut == 0.0) or v > threshold:
            selected += 1
    if (abs_cut == 0.0 and rel_cut == 0.0 and max_bond < count
            and singular[max_bond] > 64.0 * EPS * count * singular[0]):
        return -2
    return max(1, min(max_bond, selected))


def direct_svd_factors(m_mat, max_bond, abs_cut=0.0, rel_cut=0.0):
    """``singleGpuSvdFactors`` (dist_svd.cuh:233-283): left = U_k, right = S_k Vh_k."""
    u, s, vh = np.linalg.svd(m_mat, full_matrices=False)
    k = select_rank(s, max_bond, abs_cut, rel_cut)
    if k == -2:
        raise InsufficientBond(f"max bond {max_bond} is insufficient for zero-cutoff simulation")
    if k < 1:
        raise NonfiniteSvd("direct MPS SVD produced nonfinite singular values")
    return u[:, :k], s[:k, None] * vh[:k, :], s


def gate4_cx(control_left: bool) -> np.ndarray:
    """4x4 row-major [(I*2+J)*4 + (i*2+j)] of a CX (simulator_mps_dist.cu:376-384)."""
    g = np.zeros((4, 4), dtype=complex)
    for i in range(2):
        for j in range(2):
            if control_left:
                g[i * 2 + (j ^ i), i * 2 + j] = 1
            else:
                g[(i ^ j) * 2 + j, i * 2 + j] = 1
    return g


def apply2q(sites, s, g4, max_bond, abs_cut=0.0, rel_cut=0.0):
    """``apply2q`` (sharded_mps.cuh:477-516) + ``k_buildM`` (:30-45)."""
    a, b = sites[s], sites[s + 1]
    dl, dr = a.shape[0], b.shape[2]
    ab = np.einsum("lic,cjr->lijr", a, b)
    g = g4.reshape(2, 2, 2, 2)                         # [I,J,i,j]
    theta = np.einsum("IJij,lijr->lIJr", g, ab).reshape(2 * dl, 2 * dr)
    left, right, _ = direct_svd_factors(theta, max_bond, abs_cut, rel_cut)
    k = left.shape[1]
    sites[s] = left.reshape(dl, 2, k)
    sites[s + 1] = right.reshape(k, 2, dr)


def svd_evolve(spec, x, max_bond, abs_cut=0.0, rel_cut=0.0):
    """State preparation of the backend: 1q gates in place, adjacent CX by SVD.

    Site index = qubit index here; the backend's msb site map conv(q)=n-1-q
    (simulator_mps_dist.cu:387) mirrors the chain and leaves every expectation
    unchanged. Non-adjacent pairs are routed with SWAPs exactly like
    ``applyTwoQubit`` (sharded_mps.cuh:565-572).
    """
    n = spec["n"]
    vec = np.array(INITIAL_VECTORS[spec.get("initial")], dtype=complex)
    sites = [vec.reshape(1, 2, 1).copy() for _ in range(n)]
    swap = np.zeros((4, 4), dtype=complex)
    for i in range(2):
        for j in range(2):
            swap[j * 2 + i, i * 2 + j] = 1
    for op in spec["ops"]:
        if op[0] == "cx":
            c, t = op[1], op[2]
            lo, hi = min(c, t), max(c, t)
            g = gate4_cx(c == lo)
            for pos in range(hi, lo + 1, -1):
                apply2q(sites, pos - 1, swap, max_bond, abs_cut, rel_cut)
            apply2q(sites, lo, g, max_bond, abs_cut, rel_cut)
            for pos in range(lo + 1, hi):
                apply2q(sites, pos, swap, max_bond, abs_cut, rel_cut)
        else:
            q = op[1]
            sites[q] = np.einsum("ij,ajb->aib", op_matrix(op, x), sites[q])
    return sites


def allocation_bonds(n, edges, max_bond):
    """Predicted bond dims, matching graph_resources.allocation_bound (:12-32)."""
    bonds = [1] * (n + 1)
    for a, b in edges:
        a, b = sorted((a, b))
        for cut in [*range(b - 1, a, -1), a, *range(a + 1, b)]:
            bonds[cut + 1] = min(2 * bonds[cut], 2 * bonds[cut + 2], max_bond)
    return bonds


def right_identity_envs(sites):
    """R_q[b,b'] = sum conj(A[b,i,c]) A[b',i,c'] R_{q+1}[c,c'], R_n = 1.

    Same recursion as k_rightStage/k_rightFinish (sharded_mps.cuh:61-90) in
    the bra/ket orientation of the left transfer.
    """
    n = len(sites)
    r = [None] * (n + 1)
    r[n] = np.ones((1, 1), dtype=complex)
    for q in range(n - 1, -1, -1):
        a = sites[q]
        r[q] = np.einsum("bic,cd,eid->be", a.conj(), r[q + 1], a)
    return r


def reverse_chain(sites):
    """The same state with the chain read backwards: site s <- site n-1-s, bonds swapped.

    This is the plugin's msb layout (site = n-1-qubit) of a qubit-ordered MPS."""
    return [np.transpose(a, (2, 1, 0)).copy() for a in reversed(sites)]


def statevector(sites):
    """Dense amplitudes, qubit 0 = most significant (ShardedMPS::toStatevector order)."""
    psi = sites[0].reshape(2, -1)
    for a in sites[1:]:
        psi = np.einsum("xc,cjr->xjr", psi, a).reshape(-1, a.shape[2])
    return psi.reshape(-1)


def dense_statevector(spec, x):
    """Independent dense simulation (test_reverse_mps.py:54-71 pattern), q0 most significant."""
    n = spec["n"]
    vec = np.array(INITIAL_VECTORS[spec.get("initial")], dtype=complex)
    state = vec
    for _ in range(n - 1):
        state = np.kron(state, vec)
    state = state.reshape([2] * n)
    for op in spec["ops"]:
        if op[0] == "cx":
            c, t = op[1], op[2]
            state = state.copy()
            idx = [slice(None)] * n
            idx[c] = 1
            sub = state[tuple(idx)]
            tax = t - (1 if t > c else 0)
            state[tuple(idx)] = np.flip(sub, axis=tax)
        else:
            m = op_matrix(op, x)
            state = np.moveaxis(np.tensordot(m, state, axes=([1], [op[1]])), 0, op[1])
    return state.reshape(-1)


def dense_expectations(psi, words):
    n = len(words[0]) if words else 0
    out = []
    for w in words:
        v = psi.reshape([2] * n)
        for q, p in enumerate(w):
            if p != "I":
                v = np.moveaxis(np.tensordot(PAULI[p], v, axes=([1], [q])), 0, q)
        out.append(np.vdot(psi, v.reshape(-1)))
    return np.array(out)


# ---------------------------------------------------------------------------
# Sampling (sharded_mps.cuh:103-188, 838-877, 986-1035) and seeds
# ---------------------------------------------------------------------------

MASK64 = (1 << 64) - 1


def sample_hash(x: int) -> int:
    """SplitMix64 finaliser ``sampleHash`` (sharded_mps.cuh:147-152)."""
    x = (x + 0x9E3779B97F4A7C15) & MASK64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & MASK64
    return x ^ (x >> 31)


def hash_uniform(seed: int, site: int, shot: int) -> float:
    """Uniform draw of ``k_chooseSample`` (sharded_mps.cuh:167-170)."""
    raw = sample_hash(((seed & 0xFFFFFFFF) << 32) ^ (site << 20) ^ shot)
    return (raw >> 11) * 2.0 ** -53


def seed_for_word(evaluation_seed: int, word: str) -> int:
    """FNV-1a ``hbatchSeedForWord`` (simulator_mps_dist.cu:586-594), site-order word."""
    h = (2166136261 ^ evaluation_seed) & 0xFFFFFFFF
    for ch in word.encode():
        h ^= ch
        h = (h * 16777619) & 0xFFFFFFFF
    return h


def seed_for_shot_shard(evaluation_seed: int, worker: int) -> int:
    """``hbatchSeedForShotShard`` (simulator_mps_dist.cu:596-608)."""
    v = (evaluation_seed + ((0x9E3779B9 * (worker + 1)) & 0xFFFFFFFF)) & 0xFFFFFFFF
    v ^= v >> 16
    v = (v * 0x7FEB352D) & 0xFFFFFFFF
    v ^= v >> 15
    v = (v * 0x846CA68B) & 0xFFFFFFFF
    v ^= v >> 16
    return v


PHILOX_M0, PHILOX_M1 = 0xD2511F53, 0xCD9E8D57
PHILOX_W0, PHILOX_W1 = 0x9E3779B9, 0xBB67AE85


def philox4x32(counter, key, rounds=10):
    """Philox4x32-10 (Salmon et al., SC'11), one block of four 32-bit words."""
    c = [v & 0xFFFFFFFF for v in counter]
    k0, k1 = key[0] & 0xFFFFFFFF, key[1] & 0xFFFFFFFF
    for r in range(rounds):
        p0 = PHILOX_M0 * c[0]
        p1 = PHILOX_M1 * c[2]
        c = [((p1 >> 32) ^ c[1] ^ k0) & 0xFFFFFFFF, p1 & 0xFFFFFFFF,
             ((p0 >> 32) ^ c[3] ^ k1) & 0xFFFFFFFF, p0 & 0xFFFFFFFF]
        if r != rounds - 1:
            k0 = (k0 + PHILOX_W0) & 0xFFFFFFFF
            k1 = (k1 + PHILOX_W1) & 0xFFFFFFFF
    return c


def philox_uniform(seed: int, site: int, shot: int) -> float:
    """Engine's Philox draw: counter (shot, site, 0, 0), key (seed lo, seed hi)."""
    w = philox4x32([shot, site, 0, 0], [seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF])
    return (((w[0] << 21) ^ (w[1] >> 11)) & ((1 << 53) - 1)) * 2.0 ** -53


def sample_bits(sites, shots, seed, rng="splitmix"):
    """Perfect (Ferris-Vidal) sampling with the GPU kernels' semantics.

    Returns (bits[shots, n] of 0/1 in site order, probabilities of each choice).
    Per site: w_i = v A_i, p_i = Re(w_i R_{k+1} w_i^H) clipped at 0, bit = u < p0/(p0+p1),
    v = w_bit / sqrt(p_bit) (k_sampleW/k_sampleProbabilities/k_chooseSample).
    """
    n = len(sites)
    # right envs in k_rightFinish orientation: R[a,a'] = sum A[a,i,b] R[b,b'] conj(A[a',i,b'])
    right = [None] * (n + 1)
    right[n] = np.ones((1, 1), dtype=complex)
    for k in range(n - 1, -1, -1):
        a = sites[k]
        right[k] = np.einsum("aib,bc,dic->ad", a, right[k + 1], a.conj())
    uniform = hash_uniform if rng == "splitmix" else philox_uniform
    bits = np.zeros((shots, n), dtype=np.uint8)
    for shot in range(shots):
        v = np.ones(1, dtype=complex)
        for k in range(n):
            a = sites[k]
            w = np.einsum("a,aib->ib", v, a)
            r = right[k + 1]
            p = [max(float(np.real(np.sum(w[i] * (r @ w[i].conj())))), 0.0) for i in range(2)]
            tot = p[0] + p[1]
            if tot <= 0.0:
                p = [0.5, 0.5]
                tot = 1.0
            u = uniform(seed, k, shot)
            sel = 0 if u < p[0] / tot else 1
            bits[shot, k] = sel
            norm = 1.0 / math.sqrt(p[sel]) if p[sel] > 0.0 else 1.0
            v = w[sel] * norm
    return bits


def exact_probabilities(sites):
    """|psi|^2 over all bitstrings (site 0 most significant); small n only."""
    psi = statevector(sites)
    return np.abs(psi) ** 2


def z_sample_sums(bits, words):
    """``k_zSampleSums`` (sharded_mps.cuh:193-214): sum over shots of (-1)^parity."""
    sums = []
    for w in words:
        mask = np.array([c == "Z" for c in w])
        parity = bits[:, mask].astype(np.int64).sum(axis=1) & 1
        sums.append(int(np.sum(1 - 2 * parity)))
    return np.array(sums, dtype=np.int64)


# ---------------------------------------------------------------------------
# Helpers for word formats
# ---------------------------------------------------------------------------

def qubit_words_to_site_words(words):
    """The backend reverses each CUDA-Q word so site = n-1-qubit (simulator:571-583)."""
    return [w[::-1] for w in words]


def counts_from_bits(bits):
    """CUDA-Q counts keys: q0 leftmost (sharded_mps.cuh:896-899), bits in qubit order."""
    out = {}
    for row in bits:
        key = "".join("1" if b else "0" for b in row)
        out[key] = out.get(key, 0) + 1
    return out
