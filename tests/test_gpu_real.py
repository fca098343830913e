"""GPU: the real-arithmetic trie levels (variant "real_pf") for circuits of real
gates. Environments are carried as real parts with the plan's Y-count phase;
results must equal the reference's ReverseMPS golden energies (1e-9 relative)
on every real-gate circuit, including words with X and Y, equal the complex
DMMA kernels to rounding on the benchmark batch (energies 1e-11 relative,
per-term values 1e-12), in both the prefix and the split evaluation; complex
circuits refuse the variant and the autotuner never picks it for them."""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "reverse_mps_golden.json").read_text())
LARGE = json.loads((Path(__file__).parent / "golden" / "large_workloads_golden.json").read_text())
REAL_GATES = {"ry", "cx", "x", "z", "h", "swap"}


def _real(case):
    return all(op[0] in REAL_GATES for op in case["spec"]["ops"])


def _spec(case):
    s = case["spec"]
    return dict(n=s["n"], ops=[tuple(o) for o in s["ops"]], initial=s["initial"], count=s["count"])


@pytest.fixture(scope="module")
def vq(cuda_device):
    import vqemps
    return vqemps


@pytest.mark.parametrize("split", ["auto", "off", "on"])
@pytest.mark.parametrize("order", ["msb", "qubit"])
@pytest.mark.parametrize("case", [c for c in GOLDEN if _real(c)], ids=lambda c: c["name"])
def test_real_levels_match_reference_golden(vq, case, order, split):
    eng = vq.Engine(0, 16)
    eng.set_split_mode({"auto": None, "off": False, "on": True}[split])
    eng.set_spec(_spec(case), site_order=order)
    eng.set_level_variant("real_pf")
    ham = eng.set_hamiltonian(case["words"], case["coeffs"])
    e = float(eng.energy(ham, np.array(case["x"]))[0])
    assert abs(e - case["energy"]) <= 1e-9 * max(1.0, abs(case["energy"]))
    eng.close()


@pytest.mark.parametrize("case", [c for c in GOLDEN if not _real(c)], ids=lambda c: c["name"])
def test_complex_circuits_refuse_real_levels(vq, case):
    eng = vq.Engine(0, 16)
    eng.set_spec(_spec(case))
    ham = eng.set_hamiltonian(case["words"], case["coeffs"])
    eng.set_level_variant("real_pf")
    with pytest.raises(vq.EngineError, match="real gates"):
        eng.energy(ham, np.array(case["x"]))
    eng.set_level_variant(None)
    e = float(eng.energy(ham, np.array(case["x"]))[0])
    assert abs(e - case["energy"]) <= 1e-9 * max(1.0, abs(case["energy"]))
    assert eng.level_variant(ham, 1) != "real_pf"
    eng.close()


def test_real_levels_with_x_and_y_words(vq):
    """H gates make X and Y expectations nonzero (even numbers of Y's); odd
    numbers of Y's vanish for real amplitudes. Per-term values against the
    complex kernel."""
    from oracle import mps_oracle as O
    n = 10
    spec = O.hardware_efficient_spec(n, 3, ("ry",), "linear")
    spec["ops"] = [("h", q) for q in range(n)] + list(spec["ops"])
    rng = np.random.default_rng(9)
    words = ["".join(rng.choice(list("IXYZ"), n, p=[0.55, 0.15, 0.15, 0.15])) for _ in range(400)]
    words += ["YY" + "I" * (n - 2), "Y" + "I" * (n - 1), "XYXYIIIIII", "IIIIIIIIII"]
    coeffs = rng.normal(size=len(words))
    x = rng.uniform(-np.pi, np.pi, (3, spec["count"]))
    out = {}
    for variant in ("real_pf", "dmma3_pf"):
        for split in (False, True):
            eng = vq.Engine(0, 16)
            eng.set_split_mode(split)
            eng.set_spec(spec)
            eng.set_level_variant(variant)
            ham = eng.set_hamiltonian(words, coeffs)
            e, pt = eng.energy(ham, torch.tensor(x, device=eng.device), per_term=True)
            out[variant, split] = (e.cpu().numpy(), pt.cpu().numpy())
            eng.close()
    ref_e, ref_pt = out["dmma3_pf", False]
    psi = O.dense_statevector(spec, x[0])
    dense = O.dense_expectations(psi, words).real
    np.testing.assert_allclose(ref_pt[0], dense, atol=1e-11)
    for key, (e, pt) in out.items():
        np.testing.assert_allclose(e, ref_e, rtol=1e-11, atol=1e-11)
        np.testing.assert_allclose(pt, ref_pt, rtol=0, atol=1e-12)
    odd = [i for i, w in enumerate(words) if w.count("Y") % 2 == 1]
    assert np.all(out["real_pf", True][1][:, odd] == 0.0)


def test_real_levels_on_the_benchmark_batch(vq):
    from vqemps import workloads as VW
    spec, words, coeffs, thetas = VW.batched_40q(seed=0, batch=256)
    g = LARGE["batched_40q"]
    out = {}
    for variant in ("real_pf", "dmma3_pf"):
        eng = vq.Engine(0, 16)
        eng.set_spec(spec)
        eng.set_level_variant(variant)
        ham = eng.set_hamiltonian(words, coeffs)
        out[variant] = eng.energy(ham, torch.tensor(thetas, device=eng.device)).cpu().numpy()
        eng.close()
    for i, ref in zip(g["indices"], g["energies"]):
        assert abs(out["real_pf"][i] - ref) <= 1e-9 * max(1.0, abs(ref))
    np.testing.assert_allclose(out["real_pf"], out["dmma3_pf"], rtol=1e-11, atol=1e-9)


@pytest.mark.parametrize("pattern", ["linear", "reverse_linear"])
@pytest.mark.parametrize("order", ["msb", "qubit"])
def test_real_gate_chain_state_equals_dense_state(vq, pattern, order):
    """The real-arithmetic Jacobi chain (selected for circuits of real gates)
    prepares the dense statevector to 1e-11, zero padding included."""
    from oracle import mps_oracle as O
    spec = O.hardware_efficient_spec(8, 3, ("ry",), pattern)
    x = np.random.default_rng(3).uniform(-np.pi, np.pi, spec["count"])
    eng = vq.Engine(0, 8)
    eng.set_spec(spec, site_order=order)
    ham = eng.set_hamiltonian(["Z" + "I" * 7], [1.0])
    eng.energy(ham, x)
    dims = eng.bond_dims()
    raw = eng.sites(0)
    assert np.all(raw.imag == 0.0)
    sites = [raw[s, :dims[s], :, :dims[s + 1]] for s in range(8)]
    if order == "msb":
        sites = O.reverse_chain(sites)
    np.testing.assert_allclose(O.statevector(sites), O.dense_statevector(spec, x), atol=1e-11)
    eng.close()


def test_real_routed_circuit_pair_equals_chain_and_dense(vq):
    """Non-adjacent CX (SWAP routing), SWAP, H, X, Z and real U1 / U2 matrices:
    the two-CTA and one-CTA real chains give the same bits, equal to the dense
    state; a state with 32-row Theta blocks goes through the real Jacobi."""
    from oracle import mps_oracle as O
    rng = np.random.default_rng(12)
    u = np.linalg.qr(rng.normal(size=(4, 4)))[0].astype(complex)
    r1 = np.linalg.qr(rng.normal(size=(2, 2)))[0].astype(complex)
    ops = [("h", 0), ("ry", 1, 0), ("cx", 0, 4), ("u2", 2, 5, u), ("ry", 4, 1), ("cx", 5, 3), ("swap", 1, 6),
           ("u1", 3, r1), ("cx", 6, 2), ("z", 0), ("x", 6), ("ry", 6, 2), ("cx", 1, 2), ("h", 3), ("cx", 0, 5),
           ("ry", 3, 3, 0.5)]
    x = rng.uniform(-np.pi, np.pi, 4)
    words = ["".join(rng.choice(list("IXYZ"), 7)) for _ in range(50)]
    coeffs = rng.normal(size=50)
    out = {}
    for mode in ("pair", "chain", "quad"):
        eng = vq.Engine(0, 16)
        eng.set_evolve_mode(mode)
        eng.set_level_variant("real_pf")
        eng.set_circuit(7, ops, site_order="msb")
        ham = eng.set_hamiltonian(words, coeffs)
        e, pt = eng.energy(ham, x, per_term=True)
        out[mode] = (e.cpu().numpy(), pt.cpu().numpy(), eng.sites(0), eng.bond_dims())
        eng.close()
    for mode in ("pair", "quad"):
        assert np.array_equal(out[mode][2], out["chain"][2]) and out[mode][3] == out["chain"][3]
        assert np.array_equal(out[mode][0], out["chain"][0])
    # the dense reference: U1 / U2 through their matrices
    psi = np.zeros(2 ** 7, dtype=complex)
    psi[0] = 1.0
    psi = psi.reshape([2] * 7)
    for op in ops:
        if op[0] == "cx" or op[0] == "swap" or op[0] == "u2":
            a, b = op[1], op[2]
            m = {"cx": np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=complex),
                 "swap": np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=complex),
                 "u2": op[3] if op[0] == "u2" else None}[op[0]]
            t = np.tensordot(m.reshape(2, 2, 2, 2), psi, axes=([2, 3], [a, b]))
            psi = np.moveaxis(t, [0, 1], [a, b])
        else:
            if op[0] == "u1":
                m = op[2]
            elif op[0] == "ry":
                ang = x[op[2]] * (op[3] if len(op) > 3 else 1.0)
                m = O.rotation("ry", ang)
            else:
                m = O.FIXED_MATRICES[op[0]]
            psi = np.moveaxis(np.tensordot(m, psi, axes=([1], [op[1]])), 0, op[1])
    dense = O.dense_expectations(psi.reshape(-1), words).real
    np.testing.assert_allclose(out["pair"][1][0], dense, atol=1e-11)



def test_quad_chain_equals_pair_and_chain_on_the_benchmark_circuit(vq):
    """Four CTAs per state (up to four gates per step) on the 40-qubit benchmark
    circuit: the states of 16 parameter sets equal the two-CTA and one-CTA chains'
    bit for bit, and so do the energies."""
    from vqemps import workloads as VW
    spec, words, coeffs, thetas = VW.batched_40q(seed=0, batch=16)
    out = {}
    for mode in ("quad", "pair", "chain"):
        eng = vq.Engine(0, 16)
        eng.set_evolve_mode(mode)
        eng.set_spec(spec)
        eng.set_level_variant("real_pf")
        ham = eng.set_hamiltonian(words, coeffs)
        e = eng.energy(ham, torch.tensor(thetas, device=eng.device)).cpu().numpy()
        out[mode] = (e, [eng.sites(b) for b in (0, 7, 15)], eng.bond_dims())
        eng.close()
    for mode in ("pair", "chain"):
        assert np.array_equal(out["quad"][0], out[mode][0])
        assert all(np.array_equal(a, c) for a, c in zip(out["quad"][1], out[mode][1]))
        assert out["quad"][2] == out[mode][2]


def test_real_site_gradient_kernels_equal_four_product_kernels(vq):
    """For a circuit of real gates the default gradient variant runs the real-site
    level kernels (the products with a site tile drop the terms of its zero
    imaginary parts): energies and gradients equal the four-product DMMA
    variant's bit for bit, with the split plan and checkpointing."""
    from vqemps import workloads as VW
    spec, words, coeffs, thetas = VW.batched_40q(seed=4, batch=3, terms=1500)
    out = {}
    for variant in ("dmma3", "dmma"):
        eng = vq.Engine(0, 16)
        eng.set_spec(spec)
        eng.set_grad_variant(variant)
        eng.set_grad_checkpoint(4)
        ham = eng.set_hamiltonian(words, coeffs)
        e, g = eng.energy_grad(ham, torch.tensor(thetas, device=eng.device))
        out[variant] = (e.cpu().numpy(), g.cpu().numpy(), eng.plan_stats(ham)["cut"])
        eng.close()
    assert out["dmma3"][2] >= 1
    assert np.array_equal(out["dmma3"][0], out["dmma"][0])
    assert np.array_equal(out["dmma3"][1], out["dmma"][1])
