"""Learned warm start: training data from plain-method solves, training on the
GPU with the network's own kernels, and the time-to-same-energy comparison.

  python -m vqemps.warmstart generate --count 1000 --out solves.npz
  python -m vqemps.warmstart train --data solves.npz --out params.npz
  python -m vqemps.warmstart evaluate --params params.npz --count 20

The plain method is ``strategy.IndependentPartitionVQE`` (partition warm start,
local solves, one global L-BFGS-B refinement). The learned method replaces the
partition warm start by the network's proposal and runs the same global
refinement from it. Every proposal is judged by the exact MPS energy, in one
batched call with the all-zero angles (the |0...0> product state, the ansatz's
trivial point): the refinement starts from whichever of the two is lower, and
the partition warm start runs instead when the proposal's energy is not finite.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np
import torch

from . import mpnn as M
from ._lib import EngineError
from .strategy import GlobalProblem, IndependentPartitionVQE
from . import workloads as WL

LAYERS = 5          # reps 4 + final rotation layer: angles per qubit


def theta_to_angles(theta, n, layers=LAYERS):
    """(layer, qubit) parameter order -> [n, layers], wrapped to (-pi, pi]."""
    a = np.asarray(theta, dtype=np.float64).reshape(layers, n).T
    return np.pi - np.mod(np.pi - a, 2 * np.pi)


def angles_to_theta(angles):
    return np.ascontiguousarray(np.asarray(angles, dtype=np.float64).T.reshape(-1))


def canonical_angles(mag, layers=LAYERS):
    """Training target of a solve: the product state with the solve's
    magnetizations <Z_q>. Rotation layers 0..L-2 are zero (the CX chains then act
    on |0...0> and change nothing) and the last layer is arccos(<Z_q>), so
    <Z_q> = cos(theta_q) exactly. Raw solve angles are not a learnable target:
    a seeded random start lands on one of many equivalent angle sets."""
    mag = np.clip(np.asarray(mag, dtype=np.float64), -1.0, 1.0)
    out = np.zeros((mag.size, layers))
    out[:, -1] = np.arccos(mag)
    return out


def magnetizations(engine, n, theta):
    """<Z_q> of the ansatz state at theta (the engine holds the n-qubit circuit)."""
    words = ["I" * q + "Z" + "I" * (n - q - 1) for q in range(n)]
    h = engine.set_hamiltonian(words, np.ones(n))
    _, pt = engine.energy(h, torch.as_tensor(np.atleast_2d(theta), dtype=torch.float64, device=engine.device),
                          per_term=True)
    engine.free_hamiltonian(h)
    return pt[0].cpu().numpy()


class _TargetReached(Exception):
    pass


def solve_plain(engine, n, words, coeffs, *, block_maxiter=30, global_maxiter=10, energy_tol=1.0, seed=0):
    """One plain-method solve; returns (result dict with wall times, strategy)."""
    t0 = time.perf_counter()
    strat = IndependentPartitionVQE(engine, n, words, coeffs, block_maxiter=block_maxiter,
                                    global_maxiter=global_maxiter, energy_tol=energy_tol, seed=seed)
    out = strat.run()
    out["wall_s"] = time.perf_counter() - t0
    out["setup_s"] = out["wall_s"] - out["total_s"]
    return out, strat


class LearnedWarmStart:
    """Network proposal -> exact energy check -> global L-BFGS-B refinement."""

    def __init__(self, engine, params, device=0):
        self.engine = engine
        self.net = M.MPNN(device, params=params)

    def propose(self, n, words, coeffs):
        batch = M.make_batch([M.graph_features(n, words, coeffs)], self.net.device)
        ang = self.net.forward(batch).double().cpu().numpy()
        return angles_to_theta(ang)

    def run(self, n, words, coeffs, *, global_maxiter=10, energy_tol=1.0, target=None):
        """Propose, judge, refine. ``target``: stop as soon as an evaluated
        energy is <= target (time-to-same-energy)."""
        t0 = time.perf_counter()
        # the global problem only: the learned path needs no partition plan
        strat = GlobalProblem(self.engine, n, words, coeffs, energy_tol=energy_tol)
        t_setup = time.perf_counter() - t0
        P = strat.num_params
        theta = self.propose(n, words, coeffs)
        t_prop = time.perf_counter() - t0
        try:
            e_prop, e_zero = (float(v) for v in strat.energy(np.stack([theta, np.zeros(P)])))
        except EngineError:      # the proposal's state failed (nonfinite angles or SVD)
            e_prop, e_zero = float("nan"), float(strat.energy(np.zeros((1, P)))[0])
        fallback = not np.isfinite(e_prop)
        start = "proposal"
        if not fallback and e_zero < e_prop:
            start, theta = "zero", np.zeros(P)
        trace = []

        def watch(e):
            trace.append((time.perf_counter() - t0, float(e)))
            if target is not None and e <= target:
                raise _TargetReached()

        reached = None
        try:
            watch(min(e_prop, e_zero) if not fallback else e_prop)
            if fallback:
                plain, _ = solve_plain(self.engine, n, words, coeffs, global_maxiter=global_maxiter,
                                       energy_tol=energy_tol)
                return dict(fallback=True, start="partition", proposal_energy=e_prop, zero_energy=e_zero,
                            best_energy=plain["best_energy"], best_params=plain["best_params"], reached_s=None,
                            wall_s=time.perf_counter() - t0)
            base_energy, base_vg = strat.energy, strat.value_grad

            def energy(th):
                e = base_energy(th)
                watch(e[0])
                return e

            def value_grad(th):
                e, g = base_vg(th)
                watch(e)
                return e, g

            strat.energy, strat.value_grad = energy, value_grad
            res = strat.refine(theta, global_maxiter)
            best = res["energy"]
        except _TargetReached:
            reached = trace[-1][0]
            best = trace[-1][1]
        return dict(fallback=False, start=start, proposal_energy=e_prop, zero_energy=e_zero, proposal_s=t_prop,
                    setup_s=t_setup,
                    best_energy=min(best, min(e for _, e in trace)), reached_s=reached,
                    wall_s=time.perf_counter() - t0, trace=trace)


# ---------------------------------------------------------------------------
# training data and training
# ---------------------------------------------------------------------------
def generate(count, out, seed0=1000, nmin=16, nmax=48, log_every=50):
    from .engine import Engine
    eng = Engine(0, 16)
    rows = dict(seed=[], n=[], T=[], warm=[], best=[], wall=[], angles=[], mag=[])
    t_start = time.perf_counter()
    for i in range(count):
        seed = seed0 + i
        n, words, coeffs = WL.warm_start_problem(seed, nmin, nmax)
        res, _ = solve_plain(eng, n, words, coeffs)
        rows["seed"].append(seed)
        rows["n"].append(n)
        rows["T"].append(len(words))
        rows["warm"].append(res["warm_start_energy"])
        rows["best"].append(res["best_energy"])
        rows["wall"].append(res["wall_s"])
        rows["angles"].append(theta_to_angles(res["best_params"], n).astype(np.float32))
        rows["mag"].append(magnetizations(eng, n, res["best_params"]).astype(np.float32))
        if log_every and (i + 1) % log_every == 0:
            print(json.dumps(dict(solves=i + 1, elapsed_s=time.perf_counter() - t_start)), flush=True)
    np.savez_compressed(out, seed=np.array(rows["seed"]), n=np.array(rows["n"]), T=np.array(rows["T"]),
                        warm=np.array(rows["warm"]), best=np.array(rows["best"]), wall=np.array(rows["wall"]),
                        angles=np.concatenate(rows["angles"]), mag=np.concatenate(rows["mag"]))
    return out


def load_dataset(paths, nmin=16, nmax=48):
    """Graphs and canonical targets of one or more ``generate`` outputs (the
    Hamiltonians are regenerated from their seeds)."""
    graphs, targets = [], []
    for path in ([paths] if isinstance(paths, (str, Path)) else paths):
        d = np.load(path)
        off = 0
        for seed, n in zip(d["seed"], d["n"]):
            n_, words, coeffs = WL.warm_start_problem(int(seed), nmin, nmax)
            assert n_ == n
            graphs.append(M.graph_features(int(n), words, coeffs))
            targets.append(canonical_angles(d["mag"][off:off + n]).astype(np.float32))
            off += n
    return graphs, targets


def train(data, out, epochs=200, batch_graphs=32, lr=2e-3, seed=0, holdout=0.1, log_every=10):
    graphs, targets = load_dataset(data)
    rng = np.random.default_rng(seed)
    order = rng.permutation(len(graphs))
    nval = max(1, int(holdout * len(graphs)))
    val, tr = order[:nval], order[nval:]
    net = M.MPNN(0, seed=seed)
    dev = net.device

    def batch_of(idx):
        b = M.make_batch([graphs[i] for i in idx], dev)
        t = torch.tensor(np.concatenate([targets[i] for i in idx]), device=dev)
        return b, t

    val_batch = batch_of(val)
    train_batches = [batch_of(tr[i:i + batch_graphs]) for i in range(0, len(tr), batch_graphs)]
    history = []
    t0 = time.perf_counter()
    for ep in range(epochs):
        tot = 0.0
        for k in rng.permutation(len(train_batches)):
            b, t = train_batches[k]
            tot += net.train_step(b, t, lr=lr * 0.5 * (1 + np.cos(np.pi * ep / epochs))).item()
        if ep % log_every == 0 or ep == epochs - 1:
            net.forward(val_batch[0])
            vl, _ = net.loss(val_batch[1])
            history.append(dict(epoch=ep, train=tot / len(train_batches), val=vl.item(),
                                elapsed_s=time.perf_counter() - t0))
            print(json.dumps(history[-1]), flush=True)
    params = net.params()
    np.savez_compressed(out, params=params, history=json.dumps(history))
    return params, history


def evaluate(params_path, count=20, seed0=900000, n=96, terms=40000, global_maxiter=10):
    """Plain method vs learned warm start on unseen Hamiltonians: time for the
    learned path to reach the plain method's final energy (+-1e-4 relative)."""
    from .engine import Engine
    params = np.load(params_path)["params"]
    eng = Engine(0, 16)
    learned = LearnedWarmStart(eng, params)
    rows = []
    for i in range(count):
        nn, words, coeffs = WL.warm_start_test_problem(seed0 + i, n, terms)
        plain, strat = solve_plain(eng, nn, words, coeffs, global_maxiter=global_maxiter)
        e_plain = plain["best_energy"]
        target = e_plain + 1e-4 * abs(e_plain)
        lw = learned.run(nn, words, coeffs, global_maxiter=global_maxiter, target=target)
        row = dict(seed=seed0 + i, n=nn, terms=len(words), plain_energy=e_plain, plain_s=plain["wall_s"],
                   plain_local_s=plain["local_s"], warm_start_energy=plain["warm_start_energy"],
                   learned_fallback=lw["fallback"], learned_start=lw["start"], proposal_energy=lw["proposal_energy"],
                   zero_energy=lw["zero_energy"], learned_best=lw.get("best_energy"),
                   learned_reached_s=lw.get("reached_s"), learned_wall_s=lw["wall_s"],
                   learned_setup_s=lw.get("setup_s"), learned_proposal_s=lw.get("proposal_s"),
                   plain_setup_s=plain["setup_s"])
        row["ratio"] = (row["learned_reached_s"] / row["plain_s"]) if row["learned_reached_s"] else None
        rows.append(row)
        print(json.dumps(row), flush=True)
    ok = [r for r in rows if r["ratio"] is not None]
    summary = dict(instances=len(rows), reached=len(ok), fallback=sum(r["learned_fallback"] for r in rows),
                   started_from_zero=sum(r["learned_start"] == "zero" for r in rows),
                   median_ratio=float(np.median([r["ratio"] for r in ok])) if ok else None,
                   within_half=sum(r["ratio"] <= 0.5 for r in ok))
    print(json.dumps(dict(summary=summary)), flush=True)
    return rows, summary


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    g = sub.add_parser("generate")
    g.add_argument("--count", type=int, default=1000)
    g.add_argument("--seed0", type=int, default=1000)
    g.add_argument("--out", required=True)
    t = sub.add_parser("train")
    t.add_argument("--data", required=True, nargs="+")
    t.add_argument("--out", required=True)
    t.add_argument("--epochs", type=int, default=200)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--batch", type=int, default=32)
    e = sub.add_parser("evaluate")
    e.add_argument("--params", required=True)
    e.add_argument("--count", type=int, default=20)
    e.add_argument("--n", type=int, default=96)
    e.add_argument("--terms", type=int, default=40000)
    e.add_argument("--out")
    args = ap.parse_args(argv)
    torch.cuda.set_device(0)
    if args.cmd == "generate":
        generate(args.count, args.out, args.seed0)
    elif args.cmd == "train":
        train(args.data, args.out, epochs=args.epochs, lr=args.lr, batch_graphs=args.batch)
    else:
        rows, summary = evaluate(args.params, args.count, n=args.n, terms=args.terms)
        if args.out:
            ratios = [r["ratio"] for r in rows if r["ratio"] is not None]
            med = lambda key: float(np.median([r[key] for r in rows if r.get(key) is not None]))
            Path(args.out).write_text(json.dumps(dict(
                command=f"cd graph-vqe_b200 && python -m vqemps.warmstart evaluate --params {args.params} "
                        f"--count {args.count} --n {args.n} --terms {args.terms}",
                instances=f"{args.count} unseen Hamiltonians: vqemps.workloads.warm_start_test_problem(seed, "
                          f"n={args.n}, terms={args.terms}), seeds 900000..{900000 + args.count - 1}",
                weights=Path(args.params).name,
                summary=summary,
                ratio_percentiles={str(q): float(np.percentile(ratios, q)) for q in (10, 25, 50, 75, 90)}
                if ratios else None,
                plain_s_median=med("plain_s"), learned_reached_s_median=med("learned_reached_s"),
                learned_setup_s_median=med("learned_setup_s"),
                ratios=[round(x, 4) for x in ratios]), indent=1))


if __name__ == "__main__":
    main()
