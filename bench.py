"""Benchmark: batched MPS energy evaluations/s at 40 qubits, chi = 16.

Workload: 40 qubits, reverse_linear RY ansatz with 4 layers + final RY layer
(200 angles), 5,000-term seeded synthetic Pauli sum (weight <= 6, 90 % Z words,
20 % +-U(100, 1000) penalty coefficients), B = 256 parameter sets per step (SPSA
+-0.1 probe pairs around a seeded point). One step = prepare the 256 MPS states
(SVD gate chain) and evaluate all 5,000 terms on each: 256 energy evaluations.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl ours|reference]

N > 1 runs under torchrun: every rank evaluates its own B parameter sets on its
GPU (independent units, no data-path collective: weak scaling); the time is the
max over ranks. ``--impl reference`` times the CPU restatement of the
reference's ReverseMPS energy on the host cores (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "graph-vqe_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

METRIC = "energy evals/s at 40q chi16 (batched)"
UNIT = "evals/s"
WORKLOAD = dict(workload="40q reverse_linear RY ansatz, 4 layers + final RY (200 angles), "
                "5000-term Pauli sum (wmax 6), chi<=16, B parameter sets per step (SPSA +-0.1 probes)",
                qubits=40, terms=5000, max_bond=16, layers=4, pattern="reverse_linear")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample-seconds", type=float, default=15.0)
    return ap.parse_args()


def dist_setup(n_gpus):
    import torch
    import torch.distributed as dist
    if n_gpus > 1 or int(os.environ.get("WORLD_SIZE", "1")) > 1:
        rank = int(os.environ.get("RANK", "0"))
        local = int(os.environ.get("LOCAL_RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local) if backend == "nccl" else None)
        return rank, local, world, dist
    return 0, 0, 1, None


def max_over_ranks(value, dist, device):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, device):
    if dist is not None:
        import torch
        t = torch.zeros(1, device=device)
        dist.all_reduce(t)


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("VQEMPS_CLOCKS_FILE", f"/tmp/vqemps_clocks_{os.getpid()}.csv"))

    def start(self):
        """Start sampling every 50 ms; give nvidia-smi time to produce its first rows."""
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.5)
        except (OSError, FileNotFoundError):
            self.proc = None

    def window(self, t0, t1):
        """Timed region as wall-clock datetimes (samples outside it are dropped)."""
        self.t0, self.t1 = t0, t1

    def stop(self):
        if self.proc is None:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["clock sampling unavailable"])
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.fh.close()
        import datetime
        rows = [[c.strip() for c in r.split(",")] for r in self.path.read_text().strip().splitlines() if r.strip()]
        kept = []
        for r in rows:
            if len(r) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f")
            except ValueError:
                continue
            if getattr(self, "t0", None) is None or self.t0 <= ts <= self.t1:
                kept.append(r)
        sm = [float(r[2]) for r in kept if r[2].replace(".", "").isdigit()]
        smax = [float(r[3]) for r in kept if r[3].replace(".", "").isdigit()]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in kept:
            for name, v in zip(names, r[6:10]):
                if v.lower() == "active":
                    reasons.add(name)
        return dict(sm_mhz=float(np.median(sm)) if sm else None, sm_max_mhz=max(smax) if smax else None,
                    reasons=sorted(reasons), samples=len(kept))


def measure_fp64_peak(torch, device):
    """cuBLAS DGEMM (FP64 tensor cores) throughput, burst: the FP64 denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def profiled_traffic(variant):
    """DRAM bytes per evaluation of all trie levels of one step, as recorded from
    an ncu capture of the same kernel in profiles/level_traffic.json (a data file
    written beside the capture's summary); None for kernels without a capture."""
    path = ROOT / "profiles" / "level_traffic.json"
    if not path.exists():
        return None
    return json.loads(path.read_text()).get("bytes_per_eval", {}).get(variant)


GOLDEN = ROOT / "tests" / "golden" / "large_workloads_golden.json"


def golden_gate(eng, ham, th, words, coeffs):
    """Before timing: the timed batch's own outputs must equal the reference's.

    tests/golden/large_workloads_golden.json holds the energies the reference's
    ReverseMPS computed for four parameter sets of this exact batch (and a digest
    of the Hamiltonian). The full batch is evaluated once and those four compared
    at 1e-9 relative; any difference stops the benchmark before a line is printed."""
    from vqemps import workloads as W
    g = json.loads(GOLDEN.read_text())["batched_40q"]
    if W.workload_digest(words, coeffs) != g["digest"]:
        raise SystemExit("golden gate: the benchmark Hamiltonian differs from the recorded one")
    e = eng.energy(ham, th).cpu().numpy()
    worst = 0.0
    for i, ref in zip(g["indices"], g["energies"]):
        err = abs(float(e[i]) - ref) / max(1.0, abs(ref))
        worst = max(worst, err)
        if not err <= 1e-9:
            raise SystemExit(f"golden gate: parameter set {i}: {e[i]!r} vs reference {ref!r}")
    return dict(checked=list(g["indices"]), max_rel_err=worst, tol=1e-9)


def cpu_reference_rate(seconds, threads):
    """The oracle's restatement of the reference CPU path (ReverseMPS energy,
    128-term chunks, prefix dedupe, complex128) on a bounded sample."""
    from oracle import cpu_baseline
    return cpu_baseline.energy_rate(seconds, threads)


def run_reference(args):
    """Reference arm: the CPU restatement of the reference's energy path, each step a
    bounded sample of the workload (a fixed number of parameter sets), all host threads."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import cpu_baseline
    threads = os.cpu_count() or 1
    w = cpu_baseline.Workload(args.batch)
    dt = w.run(1, threads)                                   # warm-up; sizes a ~2 s step
    per_step = max(1, int(round(2.0 / max(dt, 1e-3))))
    for _ in range(args.warmup):
        w.run(per_step, threads)
    total = 0.0
    for _ in range(args.steps):
        total += w.run(per_step, threads)
    evals = per_step * args.steps
    value = evals / total
    line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                ms_per_step=1000.0 * total / args.steps, higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="c128", data="synthetic", impl="reference",
                config=dict(WORKLOAD, global_batch=args.batch, parallelism=f"{threads} host threads",
                            evals_per_step=per_step),
                cpu_baseline=dict(value=value, unit=UNIT, cores=threads, kind="port",
                                  sample=cpu_baseline.describe(evals, total, threads)),
                e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    rank, local, world, dist = dist_setup(args.gpus)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    import vqemps
    from vqemps import workloads as W

    spec, words, coeffs, thetas = W.batched_40q(seed=0, batch=args.batch)
    # each rank gets its own probe set: shift the SPSA center per rank
    thetas = thetas + 1e-3 * rank
    eng = vqemps.Engine(local, 16)
    eng.set_spec(spec)
    ham = eng.set_hamiltonian(words, coeffs)
    stats = eng.plan_stats(ham)
    th = torch.tensor(thetas, dtype=torch.float64, device=device)
    out = torch.empty(args.batch, dtype=torch.float64, device=device)
    stream = torch.cuda.current_stream(device)
    # correctness gate before timing: the timed batch against the reference's energies
    gate = None
    if args.batch == 256 and rank == 0:
        gate = golden_gate(eng, ham, th, words, coeffs)
    else:
        assert torch.isfinite(eng.energy(ham, th[:2])).all()

    fp64_peak = measure_fp64_peak(torch, device)

    def step():
        eng.energy(ham, th, check_status=False)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    barrier(dist, device)
    torch.cuda.synchronize()
    clocks.start()
    import datetime
    wall0 = datetime.datetime.now()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        step()
    end.record(stream)
    end.synchronize()
    clocks.window(wall0, datetime.datetime.now())
    clock_info = clocks.stop()
    barrier(dist, device)
    elapsed = start.elapsed_time(end) * 1e-3
    elapsed = max_over_ranks(elapsed, dist, device)
    evals = args.batch * args.steps * world
    value = evals / elapsed
    ms_per_step = 1000.0 * elapsed / args.steps
    eng.check_status(args.batch)

    # ---- kernel breakdown (one extra step, events between phases) ----
    from vqemps import profiling
    phases = profiling.phase_times(eng, ham, th, repeats=3)
    level_s = phases["levels_s"]
    variant = eng.level_variant(ham, args.batch)
    # executed work: the complex kernels' count (8 real flops per complex
    # multiply-add); the real-arithmetic kernel does one real multiply-add (2
    # flops) where they do a complex one
    flops_eval = stats["flops"] / 4.0 if variant == "real_pf" else stats["flops"]
    flops_step = flops_eval * args.batch
    achieved = flops_step / level_s / 1e12
    kernel = {"simt": "level_kernel (FP64 FMA pipes)", "simt_pf": "level_pf_kernel (FP64 FMA pipes, cp.async prefetch)",
              "dmma4": "level_mma_kernel<4> (FP64 DMMA tensor cores)",
              "dmma8": "level_mma_kernel<8> (FP64 DMMA tensor cores)",
              "dmma_pf": "level_mma_pf_kernel (FP64 DMMA tensor cores, cp.async parent prefetch)",
              "dmma3_pf": "level_mma3_pf_kernel (FP64 DMMA tensor cores, Gauss 3-product complex multiply, "
                          "cp.async parent prefetch)",
              "real_pf": "level_real_pf_kernel (FP64 DMMA tensor cores, real arithmetic with Y-count phases for "
                         "real-amplitude states, 1-D bulk-copy staging on mbarriers)"}.get(variant, str(variant))
    traffic = profiled_traffic(variant)
    roofline = dict(bound="tensor" if variant and variant != "simt" and variant != "simt_pf" else "fp64",
                    achieved=achieved,
                    peak=fp64_peak, unit="TFLOP/s", frac=achieved / fp64_peak,
                    traffic=traffic * args.batch if traffic else None,
                    kernel=kernel + ", all trie levels of one step",
                    peak_source="cuBLAS FP64 DGEMM 8192^3 (DMMA tensor cores) measured in this run, burst",
                    survey_unit_tflops=stats["flops_survey"] * args.batch / level_s / 1e12)

    # ---- e2e: host buffers through the C ABI, copies inside the timed region ----
    th_host = torch.tensor(thetas, dtype=torch.float64).pin_memory()
    e_host = torch.empty(args.batch, dtype=torch.float64).pin_memory()
    for _ in range(2):
        eng.energy_host(ham, th_host, e_host)
    barrier(dist, device)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.energy_host(ham, th_host, e_host)
    t1 = time.perf_counter()
    e2e_elapsed = max_over_ranks(t1 - t0, dist, device)
    e2e = dict(value=evals / e2e_elapsed, unit=UNIT, h2d_bytes_per_step=th_host.numel() * 8,
               d2h_bytes_per_step=e_host.numel() * 8 + 4 * args.batch)

    # ---- plain path: one parameter set per call, same kernels ----
    plain_n = 20
    for k in range(3):
        eng.energy(ham, th[k:k + 1], check_status=False)
    torch.cuda.synchronize()
    ps, pe = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ps.record(stream)
    for k in range(plain_n):
        eng.energy(ham, th[k:k + 1], check_status=False)
    pe.record(stream)
    pe.synchronize()
    plain_rate = plain_n / (ps.elapsed_time(pe) * 1e-3)

    cpu = None
    if rank == 0 and world == 1:
        cpu_r = cpu_reference_rate(args.cpu_sample_seconds, os.cpu_count() or 1)
        cpu = dict(value=cpu_r["value"], unit=UNIT, cores=cpu_r["threads"], kind="port", sample=cpu_r["sample"])

    if rank == 0:
        line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
                    ms_per_step=ms_per_step, higher_is_better=True, scaling="weak", vs_baseline=None,
                    dtype="f64", data="synthetic",
                    config=dict(WORKLOAD, global_batch=args.batch * world, parallelism=f"replicas x{world}",
                                l2="working set per step > L2 (level environments ~6 GB): no flush needed",
                                plain_evals_per_s=plain_rate, batched_over_plain=value / world / plain_rate,
                                flops_per_eval=flops_eval, survey_flops_per_eval=stats["flops_survey"],
                                trie_node_sites=stats["node_sites"],
                                phases_ms=phases["ms"], golden_gate=gate),
                    roofline=roofline, cpu_baseline=cpu, e2e=e2e,
                    gpu_launches=phases["launches_per_step"] * args.steps,
                    clocks=clock_info)
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
