"""Secondary workloads of the engine, timed on one GPU with CUDA events.

  python -m vqemps.benchmarks partitions   # 64 uneven partitions + 1000/4096 Philox shots
  python -m vqemps.benchmarks gradient     # 64q, 20,000 terms, B = 32 energy + gradient
  python -m vqemps.benchmarks graphs       # CUDA-graph replay vs direct launches
  python -m vqemps.benchmarks chain        # the gate chain per mode (one, two, four CTAs) and batch size

Each prints one JSON line per measurement. Inputs are the seeded synthetic
workloads of ``oracle.workloads`` (no public data set stands behind them).
Results are timed after warm-up with events on the launching stream; the
working sets exceed L2 except where a line says otherwise.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
for _p in (ROOT, ROOT / "graph-vqe_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

import vqemps  # noqa: E402
from vqemps import workloads as W  # noqa: E402


def _events_ms(fn, reps, stream):
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(reps):
        fn()
    end.record(stream)
    end.synchronize()
    return start.elapsed_time(end) / reps


def bench_partitions(reps: int = 10):
    parts = W.uneven_partitions(seed=0)
    eng = vqemps.Engine(0, 16)
    dev = eng.device
    stream = torch.cuda.current_stream(dev)
    t0 = time.perf_counter()
    ps = eng.set_partitions([(s["n"], s["ops"], w, c) for s, w, c, _ in parts])
    setup_s = time.perf_counter() - t0
    theta = ps.pack_theta([p[3] for p in parts], device=dev)
    out = torch.empty(ps.K, dtype=torch.float64, device=dev)
    shape = dict(partitions=ps.K, qubits=[min(ps.ns), max(ps.ns)], terms=[min(ps.T), max(ps.T)],
                 total_terms=int(sum(ps.T)), n_max=ps.n_max)
    for _ in range(3):
        eng.partition_energy(ps, theta, out=out, check_status=False)
    eng.check_status(ps.K)
    ms = _events_ms(lambda: eng.partition_energy(ps, theta, out=out, check_status=False), reps, stream)
    graph = eng.capture(lambda: eng.partition_energy(ps, theta, out=out, check_status=False))
    ms_graph = _events_ms(graph.replay, reps, stream)
    # plain: one engine per partition, one state per call, the same kernels
    singles = []
    for spec, words, coeffs, x in parts:
        se = vqemps.Engine(0, 16)
        se.set_spec(spec)
        se.set_level_variant("dmma3_pf")
        se.set_split_mode("off")          # the partition set's prefix plan
        singles.append((se, se.set_hamiltonian(words, coeffs),
                        torch.tensor(x, dtype=torch.float64, device=dev).unsqueeze(0),
                        torch.empty(1, dtype=torch.float64, device=dev)))

    def plain_sweep():
        for se, h, x, o in singles:
            se.energy(h, x, out=o, check_status=False)

    plain_sweep()
    torch.cuda.synchronize()
    ms_plain = _events_ms(plain_sweep, max(2, reps // 3), stream)
    line = dict(workload="uneven partitions, analytic energy", **shape, setup_s=setup_s,
                batched_ms=ms, batched_graph_ms=ms_graph, plain_sequential_ms=ms_plain,
                partitions_per_s=ps.K / (ms * 1e-3), batched_over_plain=ms_plain / ms,
                flops_per_sweep=ps.flops, levels=ps.levels)
    print(json.dumps(line), flush=True)
    for shots in (1000, 4096):
        for _ in range(2):
            eng.partition_sampled_energy(ps, theta, shots, 7, "philox", return_bits=True)
        bits = torch.empty((ps.K, shots, ps.W), dtype=torch.int64, device=dev)
        e = torch.empty(ps.K, dtype=torch.float64, device=dev)
        from .engine import _ptr, _stream

        def sampled():
            eng.lib.vqemps_partition_sampled_energy(eng.ctx, ps.handle, _ptr(theta), 1, shots, 7, 1, _ptr(e), None,
                                                    _ptr(bits), _stream(None))

        ms_s = _events_ms(sampled, reps, stream)
        # counts on the host: bits to pinned memory, one np.unique per partition
        host = torch.empty(bits.shape, dtype=torch.int64).pin_memory()
        t0 = time.perf_counter()
        host.copy_(bits)
        arr = host.numpy()
        ncounts = 0
        for k in range(ps.K):
            keys, cnt = np.unique(arr[k], axis=0, return_counts=True)
            ncounts += len(keys)
        counts_s = time.perf_counter() - t0
        line = dict(workload=f"uneven partitions, {shots} Philox shots + shot energy", **shape, shots=shots,
                    batched_ms=ms_s, shots_per_s=ps.K * shots / (ms_s * 1e-3),
                    bit_buffer_bytes=bits.numel() * 8, host_counts_ms=counts_s * 1e3,
                    distinct_bitstrings=ncounts)
        print(json.dumps(line), flush=True)


def bench_gradient(reps: int = 3, every=(8, 1), plans=("auto", "off")):
    spec, words, coeffs, thetas = W.gradient_64q(seed=0)
    for plan in plans:
        eng = vqemps.Engine(0, 16)
        eng.set_spec(spec)
        eng.set_split_mode(plan)
        ham = eng.set_hamiltonian(words, coeffs)
        stats = eng.plan_stats(ham)
        dev = eng.device
        stream = torch.cuda.current_stream(dev)
        th = torch.tensor(thetas, dtype=torch.float64, device=dev)
        B = th.shape[0]
        eng.energy(ham, th)                                    # tunes the level kernel outside the timing
        for k in every:
            eng.set_grad_checkpoint(k)
            free0 = torch.cuda.mem_get_info(dev)[0]
            eng.energy_grad(ham, th)
            torch.cuda.synchronize()
            used = free0 - torch.cuda.mem_get_info(dev)[0]
            ms = _events_ms(lambda: eng.energy_grad(ham, th), reps, stream)
            ms_e = _events_ms(lambda: eng.energy(ham, th, check_status=False), reps, stream)
            print(json.dumps(dict(workload="64q linear RY, 320 angles, 20000 terms (wmax 6), energy + gradient",
                                  batch=B, plan="split" if stats["cut"] >= 0 else "prefix", cut=stats["cut"],
                                  energy_plan_node_sites=stats["node_sites"], checkpoint_every=k, ms_per_call=ms,
                                  grads_per_s=B / (ms * 1e-3), energy_only_ms=ms_e, grad_over_energy=ms / ms_e,
                                  workspace_growth_bytes=int(used))), flush=True)
        eng.close()
        del th
        torch.cuda.empty_cache()


def bench_graphs(reps: int = 50):
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    spec, words, coeffs, x = W.plain_12q(seed=0)
    for B in (1, 16):
        eng = vqemps.Engine(0, 16)
        eng.set_spec(spec)
        ham = eng.set_hamiltonian(words, coeffs)
        th = torch.tensor(np.tile(x, (B, 1)), dtype=torch.float64, device=dev)
        out = torch.empty(B, dtype=torch.float64, device=dev)
        fn = lambda: eng.energy(ham, th, out=out, check_status=False)  # noqa: E731
        for _ in range(3):
            fn()
        ms = _events_ms(fn, reps, stream)
        g = eng.capture(fn)
        ms_g = _events_ms(g.replay, reps, stream)
        print(json.dumps(dict(workload="12q linear RY 5 layers, 300 terms", batch=B, direct_ms=ms,
                              graph_ms=ms_g, speedup=ms / ms_g)), flush=True)


def bench_chain(batches=(1, 16, 64, 128, 256), modes=("auto", "quad", "pair", "chain"), reps: int = 5,
                sample_only: bool = False):
    """The benchmark circuit's gate chain (40 qubits, 156 two-site gates) for each
    evolve mode and batch size: the prepare phase of an energy call (CUDA events
    inside the engine). ``sample_only`` runs one-shot sampling calls instead (gate
    chain, right environments, sampler: no trie-level buffers), for profilers."""
    from vqemps import profiling
    spec, words, coeffs, thetas = W.batched_40q(seed=0, batch=max(batches))
    for mode in modes:
        for B in batches:
            eng = vqemps.Engine(0, 16)
            eng.set_evolve_mode(mode)
            eng.set_spec(spec)
            th = torch.tensor(thetas[:B], device=eng.device)
            if sample_only:
                for _ in range(reps):
                    eng.sample(th, 1, 7)
                torch.cuda.synchronize()
            else:
                ham = eng.set_hamiltonian(words, coeffs)
                for _ in range(2):
                    eng.energy(ham, th)
                ph = profiling.phase_times(eng, ham, th, repeats=reps)
                print(json.dumps(dict(workload="40q reverse_linear RY, 4 layers (156 two-site gates)", mode=mode,
                                      batch=B, prepare_ms=ph["ms"]["prepare"],
                                      states_per_s=B / ph["ms"]["prepare"] * 1e3)), flush=True)
            eng.close()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("which", choices=["partitions", "gradient", "graphs", "chain", "all"])
    ap.add_argument("--reps", type=int, default=None, help="timed repetitions per measurement")
    ap.add_argument("--every", type=int, nargs="+", default=[8, 1], help="gradient checkpoint intervals")
    ap.add_argument("--plans", nargs="+", default=["auto", "off"], choices=["auto", "off", "on"],
                    help="gradient plans: split evaluation when it saves work (auto), prefix trie (off)")
    ap.add_argument("--batches", type=int, nargs="+", default=[1, 16, 64, 128, 256], help="chain: batch sizes")
    ap.add_argument("--modes", nargs="+", default=["auto", "quad", "pair", "chain"], help="chain: evolve modes")
    ap.add_argument("--sample-only", action="store_true", help="chain: one-shot sampling calls, no output")
    args = ap.parse_args(argv)
    torch.cuda.set_device(0)
    if args.which in ("partitions", "all"):
        bench_partitions(**({"reps": args.reps} if args.reps else {}))
    if args.which in ("gradient", "all"):
        bench_gradient(every=args.every, plans=args.plans, **({"reps": args.reps} if args.reps else {}))
    if args.which in ("graphs", "all"):
        bench_graphs(**({"reps": args.reps} if args.reps else {}))
    if args.which in ("chain", "all"):
        bench_chain(batches=args.batches, modes=args.modes, sample_only=args.sample_only,
                    **({"reps": args.reps} if args.reps else {}))


if __name__ == "__main__":
    main()
