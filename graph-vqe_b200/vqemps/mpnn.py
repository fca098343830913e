"""Host side of the warm-start network: coupling-graph features, graph batches
and the ctypes binding of include/vqemps_mpnn.h (kernels in csrc/mpnn.cu).

Features of a Hamiltonian sum_k c_k P_k on n qubits (words indexed by qubit):

* node q (4): slog(h_q) / 5, slog(s_q) / 10, q / (n - 1), [q is a chain end], where
  h_q is the summed coefficient of the one-body Z terms on q, s_q the summed
  |c| of every term acting on q, and slog(x) = sign(x) log(1 + |x|) keeps the
  N(0, 1) terms and the 100-1000 penalty terms on one scale;
* edge (a, b) (3): slog(J_ab) / 5, slog(w_ab) / 10, [|a - b| = 1], where J_ab is the
  summed coefficient of the two-body ZZ terms on {a, b} and w_ab the coupling
  weight of the partition graph (independent_vqe.py:62-68: summed |c| of every
  term acting on both). Edges are the coupling graph's pairs plus the ansatz
  chain's neighbours, in both directions.

The network outputs (reps + 1) angles per qubit: the RY angle of qubit q in
layer l is theta[l * n + q], the (layer, qubit, gate) order of the ansatz.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

NODE_IN = 4
EDGE_IN = 3


def slog(x):
    x = np.asarray(x, dtype=np.float64)
    return np.sign(x) * np.log1p(np.abs(x))


# fixed feature scales: slog of a coefficient sum is at most ~10 for these Hamiltonians
SCALE_FIELD, SCALE_WEIGHT = 5.0, 10.0


def graph_features(n, words, coeffs):
    """(node features [n, 4], edge index [2, E] (src, dst), edge features [E, 3]) of one Hamiltonian."""
    coeffs = np.asarray(coeffs, dtype=np.float64)
    T = len(words)
    if T:
        arr = np.frombuffer("".join(words).encode("ascii"), dtype=np.uint8).reshape(T, n)
    else:
        arr = np.full((0, n), ord("I"), dtype=np.uint8)
    act = arr != ord("I")
    isz = arr == ord("Z")
    # active (term, qubit) pairs in row-major order: each term's qubits are
    # contiguous and ascending, starting at first[t]
    rows, cols = np.nonzero(act)
    weight = np.bincount(rows, minlength=T)
    nz = np.bincount(rows, weights=isz[rows, cols], minlength=T)
    first = np.cumsum(weight) - weight
    absc = np.abs(coeffs)
    # per-qubit sums of |c| accumulate in term order, as an axis-0 sum does
    s = np.bincount(cols, weights=absc[rows], minlength=n) if T else np.zeros(n)
    one = (weight == 1) & (nz == 1)
    h = np.zeros(n)
    if one.any():
        h = np.bincount(cols[first[one]], weights=coeffs[one], minlength=n)
    # pair sums over every pair of active qubits of every term, one weight class at
    # a time; each cell accumulates its contributions in this order, in one
    # bincount over the concatenated (cell, value) lists
    zz = (weight == 2) & (nz == 2)
    w_cells, w_vals, j_cells, j_vals = [], [], [], []
    for wgt in np.unique(weight[weight >= 2]):
        sel = np.nonzero(weight == wgt)[0]
        q = cols[first[sel][:, None] + np.arange(wgt)[None, :]]   # active qubits, ascending per term
        for i in range(wgt):
            for j in range(i + 1, wgt):
                w_cells.append(q[:, i] * n + q[:, j])
                w_vals.append(absc[sel])
        if wgt == 2:
            z = zz[sel]
            j_cells.append(q[z, 0] * n + q[z, 1])
            j_vals.append(coeffs[sel][z])

    def cell_sums(cells, vals):
        if not cells:
            return np.zeros((n, n))
        return np.bincount(np.concatenate(cells), weights=np.concatenate(vals), minlength=n * n).reshape(n, n)

    Wt = cell_sums(w_cells, w_vals)
    Jm = cell_sums(j_cells, j_vals)
    pairs = set(zip(*np.nonzero(np.triu(Wt, 1) > 0))) | {(q, q + 1) for q in range(n - 1)}
    pairs = sorted((int(a), int(b)) for a, b in pairs)
    node = np.stack([slog(h) / SCALE_FIELD, slog(s) / SCALE_WEIGHT, np.arange(n) / max(n - 1, 1),
                     ((np.arange(n) == 0) | (np.arange(n) == n - 1)).astype(float)], axis=1)
    pa = np.array(pairs, dtype=np.int64).reshape(-1, 2)
    jv = Jm[pa[:, 0], pa[:, 1]]
    f = np.stack([slog(jv) / SCALE_FIELD, slog(Wt[pa[:, 0], pa[:, 1]]) / SCALE_WEIGHT,
                  (pa[:, 1] - pa[:, 0] == 1).astype(float)], axis=1)
    src = np.stack([pa[:, 0], pa[:, 1]], axis=1).reshape(-1)
    dst = np.stack([pa[:, 1], pa[:, 0]], axis=1).reshape(-1)
    feat = np.repeat(f, 2, axis=0)
    return node.astype(np.float32), np.array([src, dst], dtype=np.int64), feat.astype(np.float32)


@dataclass
class GraphBatch:
    """Graphs concatenated into one, on the device, in the layout vqemps_graph wants."""
    n_nodes: int
    n_edges: int
    node_offsets: np.ndarray          # per graph, into the node rows
    node_feat: torch.Tensor
    edge_feat: torch.Tensor
    edge_src: torch.Tensor
    edge_dst: torch.Tensor
    dst_off: torch.Tensor
    src_perm: torch.Tensor
    src_off: torch.Tensor
    host: dict                        # host copies (for the oracle)

    def abi(self):
        g = _lib.VqempsGraph()
        g.num_nodes, g.num_edges = self.n_nodes, self.n_edges
        g.node_feat = self.node_feat.data_ptr()
        g.edge_feat = self.edge_feat.data_ptr() if self.n_edges else None
        g.edge_src = self.edge_src.data_ptr() if self.n_edges else None
        g.edge_dst = self.edge_dst.data_ptr() if self.n_edges else None
        g.dst_off = self.dst_off.data_ptr()
        g.src_perm = self.src_perm.data_ptr() if self.n_edges else None
        g.src_off = self.src_off.data_ptr()
        return g


def make_batch(graphs, device) -> GraphBatch:
    """Concatenate ``graph_features`` outputs; edges sorted by destination
    (stable), with the by-source permutation."""
    nodes, srcs, dsts, feats, offs = [], [], [], [], [0]
    for node, ei, ef in graphs:
        base = offs[-1]
        nodes.append(node)
        srcs.append(ei[0] + base)
        dsts.append(ei[1] + base)
        feats.append(ef)
        offs.append(base + node.shape[0])
    node = np.concatenate(nodes).astype(np.float32)
    src = np.concatenate(srcs).astype(np.int64)
    dst = np.concatenate(dsts).astype(np.int64)
    ef = np.concatenate(feats).astype(np.float32).reshape(-1, EDGE_IN)
    order = np.argsort(dst, kind="stable")
    src, dst, ef = src[order], dst[order], ef[order]
    N, E = node.shape[0], src.shape[0]
    dst_off = np.zeros(N + 1, dtype=np.int64)
    np.add.at(dst_off, dst + 1, 1)
    dst_off = np.cumsum(dst_off)
    perm = np.argsort(src, kind="stable")
    src_off = np.zeros(N + 1, dtype=np.int64)
    np.add.at(src_off, src + 1, 1)
    src_off = np.cumsum(src_off)
    i32 = lambda a: torch.tensor(a.astype(np.int32), device=device)  # noqa: E731
    host = dict(node=node, src=src, dst=dst, ef=ef, dst_off=dst_off, perm=perm, src_off=src_off)
    return GraphBatch(N, E, np.array(offs), torch.tensor(node, device=device), torch.tensor(ef, device=device),
                      i32(src), i32(dst), i32(dst_off), i32(perm), i32(src_off), host)


def param_shapes(width=128, layers=3, out=5, node_in=NODE_IN, edge_in=EDGE_IN):
    """Names and shapes of the flat parameter vector (include/vqemps_mpnn.h order)."""
    shapes = [("Win", (node_in, width)), ("bin", (width,))]
    for l in range(layers):
        shapes += [(f"Wm{l}", (width + edge_in, width)), (f"bm{l}", (width,)),
                   (f"Wu{l}", (2 * width, width)), (f"bu{l}", (width,))]
    shapes += [("Wo", (width, out)), ("bo", (out,))]
    return shapes


def init_params(seed=0, width=128, layers=3, out=5):
    """He-uniform weights, zero biases, a small output layer."""
    rng = np.random.default_rng(seed)
    flat = []
    for name, shape in param_shapes(width, layers, out):
        if name.startswith("b"):
            flat.append(np.zeros(shape))
        else:
            fan_in = shape[0]
            lim = np.sqrt(6.0 / fan_in) * (0.1 if name == "Wo" else 1.0)
            flat.append(rng.uniform(-lim, lim, shape))
    return np.concatenate([f.reshape(-1) for f in flat]).astype(np.float32)


class MPNN:
    """The network on one device; parameters are FP32 masters (BF16 at the MMAs)."""

    def __init__(self, device=0, width=128, layers=3, out=5, params=None, seed=0):
        self.lib = _lib.load()
        self.device = torch.device("cuda", device)
        self.width, self.layers, self.out = width, layers, out
        net = ctypes.c_void_p()
        code = self.lib.vqemps_mpnn_create(device, NODE_IN, EDGE_IN, width, layers, out, ctypes.byref(net))
        if code != 0:
            raise _lib.EngineError(code, "vqemps_mpnn_create failed")
        self.net = net
        cnt = ctypes.c_int64()
        self._check(self.lib.vqemps_mpnn_num_params(self.net, ctypes.byref(cnt)), "num_params")
        self.count = cnt.value
        self.set_params(init_params(seed, width, layers, out) if params is None else params)
        self.grad = torch.zeros(self.count, dtype=torch.float32, device=self.device)
        self.loss_buf = torch.zeros(1, dtype=torch.float32, device=self.device)

    def _check(self, code, what):
        if code != 0:
            msg = self.lib.vqemps_mpnn_last_error(self.net).decode()
            raise _lib.EngineError(code, f"{what}: {msg}")

    def close(self):
        if getattr(self, "net", None):
            self.lib.vqemps_mpnn_destroy(self.net)
            self.net = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, flat):
        flat = np.ascontiguousarray(flat, dtype=np.float32)
        if flat.size != self.count:
            raise ValueError(f"expected {self.count} parameters")
        self._check(self.lib.vqemps_mpnn_set_params(self.net, flat.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                    self.count), "set_params")

    def params(self):
        out = np.empty(self.count, dtype=np.float32)
        self._check(self.lib.vqemps_mpnn_get_params(self.net, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                    self.count), "get_params")
        return out

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def forward(self, batch: GraphBatch) -> torch.Tensor:
        """Angles [nodes, out] of every node of the batch."""
        theta = torch.empty((batch.n_nodes, self.out), dtype=torch.float32, device=self.device)
        g = batch.abi()
        self._check(self.lib.vqemps_mpnn_forward(self.net, ctypes.byref(g), ctypes.c_void_p(theta.data_ptr()),
                                                 self._stream()), "forward")
        return theta

    def backward(self, batch: GraphBatch, dtheta: torch.Tensor) -> torch.Tensor:
        g = batch.abi()
        self._check(self.lib.vqemps_mpnn_backward(self.net, ctypes.byref(g), ctypes.c_void_p(dtheta.data_ptr()),
                                                  ctypes.c_void_p(self.grad.data_ptr()), self._stream()), "backward")
        return self.grad

    def loss(self, target: torch.Tensor, weight: torch.Tensor | None = None):
        """(loss tensor [1], dloss/dtheta) of the last forward."""
        dtheta = torch.empty_like(target)
        self._check(self.lib.vqemps_mpnn_loss(self.net, ctypes.c_void_p(target.data_ptr()),
                                              ctypes.c_void_p(weight.data_ptr()) if weight is not None else None,
                                              ctypes.c_void_p(self.loss_buf.data_ptr()),
                                              ctypes.c_void_p(dtheta.data_ptr()), self._stream()), "loss")
        return self.loss_buf, dtheta

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        self._check(self.lib.vqemps_mpnn_adam_step(self.net, ctypes.c_void_p(self.grad.data_ptr()), lr, beta1,
                                                   beta2, eps, weight_decay, self._stream()), "adam")

    def train_step(self, batch: GraphBatch, target: torch.Tensor, lr=1e-3, weight=None):
        self.forward(batch)
        loss, dtheta = self.loss(target, weight)
        self.backward(batch, dtheta)
        self.adam(lr)
        return loss
