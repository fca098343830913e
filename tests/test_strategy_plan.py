"""Partition warm-start plan (CPU): simplified Hamiltonian, coupling graph,
blocks and local models against the oracle's restatement of
independent_vqe.py:53-104,140-158."""
import numpy as np
import pytest

from oracle import optim_oracle as OO
from oracle.workloads import random_hamiltonian
from vqemps.strategy import PartitionPlan, ansatz_ops, simplify


def test_simplify_merges_and_drops_zeros():
    w, c = simplify(["ZI", "IZ", "ZI", "XX", "XX"], [1.0, 2.0, 0.5, 1.0, -1.0])
    assert w == ["ZI", "IZ"] and list(c) == [1.5, 2.0]


@pytest.mark.parametrize("n,T,seed", [(30, 400, 0), (20, 150, 4), (40, 60, 7)])
def test_plan_matches_oracle(n, T, seed):
    rng = np.random.default_rng(seed)
    words, coeffs = random_hamiltonian(rng, n, T, 4)
    words.append("I" * n)
    coeffs = np.append(coeffs, 2.5)
    plan = PartitionPlan(n, words, coeffs, seed=seed)
    ow, oc = OO.simplify_terms(words, coeffs)
    assert plan.words == ow and np.array_equal(plan.coeffs, oc)
    edges = OO.coupling_edges(ow, oc)
    assert {tuple(sorted(e)) for e in plan.graph.edges} == set(edges)
    for (a, b), wgt in edges.items():
        assert plan.graph[a][b]["weight"] == pytest.approx(wgt, rel=1e-12)
    assert sorted(q for b in plan.blocks for q in b) == list(range(n))
    assert all(1 <= len(b) <= 12 for b in plan.blocks)
    models, cross = OO.local_problems(n, plan.blocks, ow, oc, 4)
    assert cross == plan.cross_terms
    for m, pm in zip(models, plan.local_models):
        assert m["terms"] == pm["terms"] and m["width"] == pm["width"] and m["constant"] == pm["constant"]
        assert list(m["parameter_indices"]) == list(pm["parameter_indices"])
    # the global parameter order is (layer, qubit, gate)
    ops, count = ansatz_ops(n, 4, ("ry",), "linear")
    assert count == plan.num_params == n * 5
    assert [o for o in ops if o[0] == "ry"][n + 3] == ("ry", 3, n + 3)


def test_disconnected_and_singleton_blocks():
    # two 3-qubit clusters and an isolated qubit: Louvain keeps the clusters apart
    words = ["ZZIIIII", "IZZIIII", "ZIZIIII", "IIIZZII", "IIIIZZI", "IIIZIZI", "IIIIIIZ"]
    plan = PartitionPlan(7, words, [1.0] * 7)
    assert plan.blocks == [[0, 1, 2], [3, 4, 5], [6]]
    single = plan.local_models[2]
    assert single["width"] == 2 and single["terms"] == [("ZI", 1.0)]
    with pytest.raises(ValueError):
        PartitionPlan(3, ["ZZI"], [1.0], blocks=[[0, 1]])
