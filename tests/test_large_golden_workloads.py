"""The benchmark-size workloads are the ones the reference's ReverseMPS was run on
(tests/golden/large_workloads_golden.json, written by make_golden.py --large):
the package generators still produce Hamiltonians with the recorded digests,
and the oracle's generators produce the same instances."""
import json
from pathlib import Path

import numpy as np

from oracle import workloads as OW
from vqemps import workloads as VW

LARGE = json.loads((Path(__file__).parent / "golden" / "large_workloads_golden.json").read_text())


def test_bench_workload_digest_matches_golden():
    spec, words, coeffs, thetas = VW.batched_40q(seed=0, batch=256)
    g = LARGE["batched_40q"]
    assert VW.workload_digest(words, coeffs) == g["digest"]
    assert len(words) == g["terms"] == 5000 and spec["n"] == g["n"] == 40
    assert thetas.shape == (256, 200)
    _, ow, oc, ot = OW.batched_40q(seed=0, batch=256)
    assert ow == words and np.array_equal(oc, coeffs) and np.array_equal(ot, thetas)


def test_gradient_workload_digest_matches_golden():
    spec, words, coeffs, thetas = VW.gradient_64q(seed=0, batch=32)
    g = LARGE["gradient_64q"]
    assert VW.workload_digest(words, coeffs) == g["digest"]
    assert len(words) == g["terms"] == 20000 and spec["n"] == g["n"] == 64
    assert thetas.shape == (32, 320)
    assert all(len(v) == 320 for v in g["gradients"])
