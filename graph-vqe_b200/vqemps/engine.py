"""Python host side of the B200 MPS engine: torch tensors in, torch tensors out.

``Engine`` owns one C-ABI context (one CUDA device). It replaces, for the VQE
hot path, the state of the reference's NVQIR plugin ``SimulatorMPSDist``
(test/backend/source/simulator_mps_dist.cu) and its per-thread workspaces.
Failures raise ``EngineError`` with the reference's messages (insufficient bond,
nonfinite SVD, invalid Pauli, unsupported gate).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import EngineError, VqempsOp, check, load


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


@dataclass
class Hamiltonian:
    """A Pauli sum loaded into an engine (words indexed by qubit)."""
    handle: int
    n: int
    T: int
    words: list
    coeffs: np.ndarray


def compile_ops(ops, n):
    """Translate an op list into the C-ABI op array and matrix table.

    Accepted ops (the ``register``/``ReverseMPS`` spec form, reverse_mps.py:12-25,
    plus the plugin's constant gates and matrices):
      (gate, q, index)  gate in rx/ry/rz, angle = theta[index]
      (gate, q, index, scale)  angle = scale * theta[index]
      (gate, q, None, angle)   constant rotation
      ('h'|'x'|'y'|'z'|'s'|'sdg', q)
      ('cx', control, target), ('swap', a, b)
      ('u1', q, 2x2 matrix), ('u2', q0, q1, 4x4 matrix)
    """
    out = []
    mats = []
    for op in ops:
        g = op[0].lower()
        o = VqempsOp()
        o.q1 = -1
        o.param = -1
        o.angle = 0.0
        o.matrix = -1
        if g in ("rx", "ry", "rz"):
            o.kind = _lib.GATES[g]
            o.q0 = int(op[1])
            if len(op) >= 3 and op[2] is not None:
                o.param = int(op[2])
                o.angle = float(op[3]) if len(op) > 3 else 1.0
            else:
                o.angle = float(op[3])
        elif g in ("h", "x", "y", "z", "s", "sdg"):
            o.kind = _lib.GATES[g]
            o.q0 = int(op[1])
        elif g in ("cx", "swap"):
            o.kind = _lib.GATES[g]
            o.q0, o.q1 = int(op[1]), int(op[2])
        elif g == "u1":
            o.kind = _lib.GATES[g]
            o.q0 = int(op[1])
            o.matrix = len(mats)
            mats.extend(np.asarray(op[2], dtype=complex).reshape(4))
        elif g == "u2":
            o.kind = _lib.GATES[g]
            o.q0, o.q1 = int(op[1]), int(op[2])
            o.matrix = len(mats)
            mats.extend(np.asarray(op[3], dtype=complex).reshape(16))
        else:
            raise EngineError(_lib.INVALID, f"unsupported gate {op[0]!r}")
        out.append(o)
    arr = (VqempsOp * max(len(out), 1))(*out)
    m = np.zeros(2 * max(len(mats), 1))
    if mats:
        z = np.asarray(mats, dtype=complex)
        m[0::2][:len(z)] = z.real
        m[1::2][:len(z)] = z.imag
    return arr, len(out), m, len(mats)


@dataclass
class PartitionSet:
    """Independent circuits of uneven width loaded into an engine together.

    ``ns[k]``/``params[k]``/``T[k]``: qubits, parameters and terms of partition
    k; parameter rows are ``P_max`` wide and per-term rows ``T_max`` wide;
    shots pack into ``W`` 64-bit words.
    """
    handle: int
    ns: list
    params: list
    T: list
    n_max: int
    P_max: int
    T_max: int
    W: int
    levels: int
    flops: float

    @property
    def K(self):
        return len(self.ns)

    def pack_theta(self, thetas, copies: int = 1, device=None):
        """Per-partition angle arrays -> the [K * copies, P_max] row layout
        (row k * copies + c; ``thetas[k]`` is [P_k] or [copies, P_k])."""
        out = torch.zeros((self.K * copies, self.P_max), dtype=torch.float64)
        for k, th in enumerate(thetas):
            t = torch.as_tensor(th, dtype=torch.float64).reshape(-1, self.params[k])
            out[k * copies:(k + 1) * copies, :self.params[k]] = t.expand(copies, -1) if t.shape[0] == 1 else t
        return out.to(device) if device is not None else out


class Engine:
    """One engine context on one CUDA device.

    ``site_order='msb'`` maps qubit q to MPS site n-1-q like the plugin
    (simulator_mps_dist.cu:387); ``'qubit'`` maps it to site q like ReverseMPS.
    Energies do not depend on the choice; SplitMix sampling reproduces the
    plugin's shots only with ``'msb'``.
    """

    def __init__(self, device: int = 0, max_bond: int = 16, abs_cut: float = 0.0,
                 rel_cut: float = 0.0):
        self.lib = load()
        self.device = torch.device("cuda", device)
        ctx = ctypes.c_void_p()
        code = self.lib.vqemps_create(device, max_bond, abs_cut, rel_cut, ctypes.byref(ctx))
        if code != _lib.OK:
            raise EngineError(code, f"vqemps_create(device={device}, max_bond={max_bond}) failed")
        self.ctx = ctx
        self.max_bond = max_bond
        self.n = 0
        self.P = 0

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.vqemps_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- circuit / Hamiltonian -------------------------------------------
    def set_circuit(self, n: int, ops, initial=None, site_order: str = "msb"):
        arr, count, mats, nm = compile_ops(ops, n)
        order = {"qubit": 0, "msb": 1}[site_order]
        mp = mats.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        check(self.ctx, self.lib.vqemps_set_circuit(self.ctx, n, arr, count, mp, nm,
                                                    _lib.INITIAL[initial], order), "set_circuit")
        p = ctypes.c_int()
        check(self.ctx, self.lib.vqemps_num_params(self.ctx, ctypes.byref(p)), "num_params")
        self.n = n
        self.P = p.value
        self.site_order = site_order

    def set_spec(self, spec, site_order: str = "msb"):
        """Load a ReverseMPS-style spec dict ``{n, ops, initial, count}``."""
        self.set_circuit(spec["n"], spec["ops"], spec.get("initial"), site_order)
        self.P = max(self.P, int(spec.get("count", self.P)))

    def bond_dims(self):
        dims = (ctypes.c_int * (self.n + 1))()
        check(self.ctx, self.lib.vqemps_bond_dims(self.ctx, dims), "bond_dims")
        return list(dims)

    def set_hamiltonian(self, words, coeffs) -> Hamiltonian:
        words = list(words)
        coeffs = np.ascontiguousarray(coeffs, dtype=np.float64)
        if len(words) != len(coeffs):
            raise EngineError(_lib.INVALID, "words and coefficients differ in length")
        for w in words:
            if len(w) != self.n:
                raise EngineError(_lib.INVALID, "Invalid analytic Pauli width")
        buf = "".join(words).encode("ascii")
        h = ctypes.c_int()
        check(self.ctx, self.lib.vqemps_set_hamiltonian(
            self.ctx, buf, coeffs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            len(words), ctypes.byref(h)), "set_hamiltonian")
        return Hamiltonian(h.value, self.n, len(words), words, coeffs)

    def free_hamiltonian(self, ham: Hamiltonian):
        check(self.ctx, self.lib.vqemps_free_hamiltonian(self.ctx, ham.handle), "free_hamiltonian")

    # "real_pf": real arithmetic, for circuits of real gates only
    LEVEL_VARIANTS = ("simt", "dmma4", "dmma8", "simt_pf", "dmma_pf", "dmma3_pf", "real_pf")

    def set_level_variant(self, variant):
        """Force a trie-level kernel (one of LEVEL_VARIANTS) or None to autotune."""
        v = -1 if variant is None else self.LEVEL_VARIANTS.index(variant)
        check(self.ctx, self.lib.vqemps_set_level_variant(self.ctx, v), "set_level_variant")

    def level_variant(self, ham: Hamiltonian, B: int):
        v = ctypes.c_int()
        check(self.ctx, self.lib.vqemps_level_variant(self.ctx, ham.handle, B, ctypes.byref(v)), "level_variant")
        return None if v.value < 0 else self.LEVEL_VARIANTS[v.value]

    def plan_stats(self, ham: Hamiltonian) -> dict:
        out = (ctypes.c_double * 10)()
        check(self.ctx, self.lib.vqemps_plan_stats(self.ctx, ham.handle, out), "plan_stats")
        keys = ("flops", "flops_survey", "node_sites", "groups", "leaves", "max_slots", "cut",
                "prefix_flops", "prefix_node_sites", "pairs")
        return dict(zip(keys, list(out)))

    def set_evolve_mode(self, mode: str):
        """Gate chain: 'quad' (four-CTA clusters, circuits of real gates; others run
        'pair'), 'pair' (two-CTA clusters on a schedule), 'chain' (one CTA, program
        order) or 'auto' (default: quad for a circuit of real gates while all its
        clusters fit the GPU at once, else pair while the batch has at most two
        states per SM, else chain). All give the same states bit for bit."""
        check(self.ctx, self.lib.vqemps_set_evolve_mode(
            self.ctx, {"chain": 0, "pair": 1, "quad": 2, "auto": -1}[mode]), "set_evolve_mode")

    def set_split_mode(self, mode):
        """Split evaluation of Hamiltonians loaded afterwards: None/'auto' (when it
        saves work), False/'off', True/'on'."""
        m = {None: -1, "auto": -1, False: 0, "off": 0, True: 1, "on": 1}[mode]
        check(self.ctx, self.lib.vqemps_set_split_mode(self.ctx, m), "set_split_mode")

    # -- helpers -------------------------------------------------------------
    def _theta(self, theta):
        t = torch.as_tensor(theta, dtype=torch.float64, device=self.device)
        if t.dim() == 1:
            t = t.unsqueeze(0)
        if t.shape[1] != self.P:
            raise EngineError(_lib.INVALID, f"expected {self.P} parameters, got {t.shape[1]}")
        return t.contiguous()

    def check_status(self, B: int, stream=None):
        st = (ctypes.c_int32 * B)()
        code = self.lib.vqemps_batch_status(self.ctx, st, B, _stream(stream))
        check(self.ctx, code, "batch")
        return list(st)

    # -- analytic energies ---------------------------------------------------
    def energy(self, ham: Hamiltonian, theta, per_term: bool = False, stream=None,
               check_status: bool = True, out=None):
        """Energies of B parameter sets (device tensors); optionally <P_k> per term.
        ``out`` (a [B] float64 device tensor) receives the energies in place."""
        t = self._theta(theta)
        B = t.shape[0]
        e = out if out is not None else torch.empty(B, dtype=torch.float64, device=self.device)
        pt = torch.empty((B, ham.T), dtype=torch.float64, device=self.device) if per_term else None
        check(self.ctx, self.lib.vqemps_energy_batch(self.ctx, ham.handle, _ptr(t), B, _ptr(e), _ptr(pt),
                                                     _stream(stream)), "energy_batch")
        if check_status:
            self.check_status(B, stream)
        return (e, pt) if per_term else e

    def energy_host(self, ham: Hamiltonian, theta_host: torch.Tensor, out_host: torch.Tensor,
                    stream=None):
        """Energies with HOST buffers (pinned CPU tensors): copies inside the call."""
        B = theta_host.shape[0]
        check(self.ctx, self.lib.vqemps_energy_batch_host(self.ctx, ham.handle, _ptr(theta_host), B,
                                                          _ptr(out_host), None, _stream(stream)),
              "energy_batch_host")
        return out_host

    def set_grad_checkpoint(self, every: int):
        """Keep every `every`-th trie level in the gradient's forward sweep (1: all)."""
        check(self.ctx, self.lib.vqemps_set_grad_checkpoint(self.ctx, int(every)), "set_grad_checkpoint")

    def set_grad_variant(self, variant: str):
        """Gradient level kernels: 'dmma3' (FP64 tensor cores, Gauss forward; default), 'dmma' or 'simt'."""
        check(self.ctx, self.lib.vqemps_set_grad_variant(self.ctx, {"simt": 0, "dmma": 1, "dmma3": 2}[variant]),
              "set_grad_variant")

    def energy_grad(self, ham: Hamiltonian, theta, stream=None):
        """Energies and dE/dtheta through the exact bond-doubling MPS."""
        t = self._theta(theta)
        B = t.shape[0]
        e = torch.empty(B, dtype=torch.float64, device=self.device)
        g = torch.empty((B, self.P), dtype=torch.float64, device=self.device)
        check(self.ctx, self.lib.vqemps_energy_grad_batch(self.ctx, ham.handle, _ptr(t), B, _ptr(e),
                                                          _ptr(g), _stream(stream)), "energy_grad_batch")
        return e, g

    def capture(self, fn, warmup: int = 2):
        """Record ``fn()`` -- engine calls on fixed device tensors, without status
        checks (they synchronise) -- into a CUDA graph and return it.

        ``fn`` runs ``warmup`` times first on a side stream, so workspaces reach
        their size and the level-kernel autotuner has decided before capture (a
        captured call may not allocate or synchronise). ``graph.replay()`` then
        re-runs every launch of the call with one submission; write new angles
        into the captured theta tensor in place between replays."""
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            for _ in range(warmup):
                fn()
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            fn()
        return graph

    # -- sampling ------------------------------------------------------------
    def sample(self, theta, shots: int, seed: int, rng: str = "splitmix", stream=None):
        """Packed bitstrings [B, shots, W] (int64 words, bit q = qubit q)."""
        t = self._theta(theta)
        B = t.shape[0]
        W = (self.n + 63) // 64
        bits = torch.empty((B, shots, W), dtype=torch.int64, device=self.device)
        check(self.ctx, self.lib.vqemps_sample(self.ctx, _ptr(t), B, shots, seed, _lib.RNG[rng], _ptr(bits),
                                               _stream(stream)), "sample")
        self.check_status(B, stream)
        return bits

    def sampled_energy(self, ham: Hamiltonian, theta, shots: int, seed: int, rng: str = "splitmix",
                       mode: str = "shared", per_term: bool = False, stream=None, check_status: bool = True):
        t = self._theta(theta)
        B = t.shape[0]
        e = torch.empty(B, dtype=torch.float64, device=self.device)
        pt = torch.empty((B, ham.T), dtype=torch.float64, device=self.device) if per_term else None
        check(self.ctx, self.lib.vqemps_sampled_energy(self.ctx, ham.handle, _ptr(t), B, shots, seed,
                                                       _lib.RNG[rng], _lib.SHOT_MODES[mode], _ptr(e),
                                                       _ptr(pt), _stream(stream)), "sampled_energy")
        if check_status:
            self.check_status(B, stream)
        return (e, pt) if per_term else e

    # -- partition sets ------------------------------------------------------
    def set_partitions(self, parts, initial=None, site_order: str = "msb") -> PartitionSet:
        """Load independent problems ``(n, ops, words, coeffs)`` as one partition set."""
        K = len(parts)
        ns = np.zeros(K, dtype=np.int32)
        op_off = np.zeros(K + 1, dtype=np.int32)
        mat_off = np.zeros(K + 1, dtype=np.int32)
        term_off = np.zeros(K + 1, dtype=np.int64)
        all_ops, all_mats, all_words, all_coeffs = [], [], [], []
        for k, (n, ops, words, coeffs) in enumerate(parts):
            arr, count, mats, nm = compile_ops(ops, n)
            words = list(words)
            if len(words) != len(coeffs):
                raise EngineError(_lib.INVALID, "words and coefficients differ in length")
            for w in words:
                if len(w) != n:
                    raise EngineError(_lib.INVALID, "Invalid analytic Pauli width")
            ns[k] = n
            all_ops.extend(arr[i] for i in range(count))
            all_mats.append(mats[:2 * nm])
            all_words.append("".join(words))
            all_coeffs.append(np.asarray(coeffs, dtype=np.float64))
            op_off[k + 1] = op_off[k] + count
            mat_off[k + 1] = mat_off[k] + nm
            term_off[k + 1] = term_off[k] + len(words)
        ops_arr = (VqempsOp * max(len(all_ops), 1))(*all_ops)
        mats = np.ascontiguousarray(np.concatenate(all_mats + [np.zeros(2)]))
        coeffs = np.ascontiguousarray(np.concatenate(all_coeffs + [np.zeros(1)]))
        buf = "".join(all_words).encode("ascii")
        order = {"qubit": 0, "msb": 1}[site_order]
        h = ctypes.c_int()
        vp = lambda a: ctypes.c_void_p(a.ctypes.data)
        check(self.ctx, self.lib.vqemps_set_partitions(
            self.ctx, K, vp(ns), ops_arr, vp(op_off), vp(mats), vp(mat_off), buf, vp(term_off), vp(coeffs),
            _lib.INITIAL[initial], order, ctypes.byref(h)), "set_partitions")
        info = np.zeros(6, dtype=np.int32)
        params = np.zeros(K, dtype=np.int32)
        flops = ctypes.c_double()
        check(self.ctx, self.lib.vqemps_partition_info(self.ctx, h.value, vp(info), vp(params),
                                                       ctypes.byref(flops)), "partition_info")
        return PartitionSet(h.value, ns.tolist(), params.tolist(), np.diff(term_off).tolist(),
                            int(info[1]), int(info[2]), int(info[3]), int(info[4]), int(info[5]),
                            flops.value)

    def free_partitions(self, pset: PartitionSet):
        check(self.ctx, self.lib.vqemps_free_partitions(self.ctx, pset.handle), "free_partitions")

    def partition_bond_dims(self, pset: PartitionSet, k: int):
        dims = (ctypes.c_int * (pset.ns[k] + 1))()
        check(self.ctx, self.lib.vqemps_partition_bond_dims(self.ctx, pset.handle, k, dims), "partition_bond_dims")
        return list(dims)

    def _part_theta(self, pset: PartitionSet, theta, copies: int):
        t = torch.as_tensor(theta, dtype=torch.float64, device=self.device)
        if t.dim() != 2 or t.shape[0] != pset.K * copies or t.shape[1] != pset.P_max:
            raise EngineError(_lib.INVALID, f"expected theta of shape [{pset.K * copies}, {pset.P_max}]")
        return t.contiguous()

    def partition_energy(self, pset: PartitionSet, theta, copies: int = 1, per_term: bool = False,
                         stream=None, check_status: bool = True, out=None):
        """Energies of ``copies`` parameter sets of every partition (state k * copies + c)."""
        t = self._part_theta(pset, theta, copies)
        B = pset.K * copies
        e = out if out is not None else torch.empty(B, dtype=torch.float64, device=self.device)
        pt = torch.empty((B, pset.T_max), dtype=torch.float64, device=self.device) if per_term else None
        check(self.ctx, self.lib.vqemps_partition_energy(self.ctx, pset.handle, _ptr(t), copies, _ptr(e),
                                                         _ptr(pt), _stream(stream)), "partition_energy")
        if check_status:
            self.check_status(B, stream)
        return (e, pt) if per_term else e

    def partition_sample(self, pset: PartitionSet, theta, shots: int, seed: int, rng: str = "philox",
                         copies: int = 1, stream=None):
        """Packed bitstrings [K * copies, shots, W] (bit q = qubit q of the state's partition)."""
        t = self._part_theta(pset, theta, copies)
        B = pset.K * copies
        bits = torch.empty((B, shots, pset.W), dtype=torch.int64, device=self.device)
        check(self.ctx, self.lib.vqemps_partition_sample(self.ctx, pset.handle, _ptr(t), copies, shots, seed,
                                                         _lib.RNG[rng], _ptr(bits), _stream(stream)),
              "partition_sample")
        self.check_status(B, stream)
        return bits

    def partition_sampled_energy(self, pset: PartitionSet, theta, shots: int, seed: int, rng: str = "philox",
                                 copies: int = 1, per_term: bool = False, return_bits: bool = False,
                                 stream=None):
        """Shot-estimated energies (one shared sample set per state), optionally the shots."""
        t = self._part_theta(pset, theta, copies)
        B = pset.K * copies
        e = torch.empty(B, dtype=torch.float64, device=self.device)
        pt = torch.empty((B, pset.T_max), dtype=torch.float64, device=self.device) if per_term else None
        bits = torch.empty((B, shots, pset.W), dtype=torch.int64, device=self.device) if return_bits else None
        check(self.ctx, self.lib.vqemps_partition_sampled_energy(
            self.ctx, pset.handle, _ptr(t), copies, shots, seed, _lib.RNG[rng], _ptr(e), _ptr(pt), _ptr(bits),
            _stream(stream)), "partition_sampled_energy")
        self.check_status(B, stream)
        out = [e]
        if per_term:
            out.append(pt)
        if return_bits:
            out.append(bits)
        return tuple(out) if len(out) > 1 else e

    def sites(self, b: int = 0, stream=None) -> np.ndarray:
        """Padded site tensors [n, 16, 2, 16] of state b of the last batch."""
        out = np.zeros(self.n * 1024, dtype=np.float64)
        check(self.ctx, self.lib.vqemps_copy_sites(self.ctx, b, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                   _stream(stream)), "copy_sites")
        z = out[0::2] + 1j * out[1::2]
        return z.reshape(self.n, 16, 2, 16)


def unpack_bits(bits: torch.Tensor, n: int) -> np.ndarray:
    """[B, shots, W] packed words -> uint8 array [B, shots, n] (qubit order)."""
    b = bits.cpu().numpy().view(np.uint64)
    q = np.arange(n)
    words = b[..., q // 64]
    return ((words >> (q % 64).astype(np.uint64)) & np.uint64(1)).astype(np.uint8)


def counts(bits: torch.Tensor, n: int, b: int = 0) -> dict:
    """CUDA-Q style counts of state b: keys have qubit 0 leftmost (sharded_mps.cuh:896-899)."""
    arr = unpack_bits(bits[b:b + 1], n)[0]
    out = {}
    for row in arr:
        key = "".join("1" if v else "0" for v in row)
        out[key] = out.get(key, 0) + 1
    return out
