"""The allocation-free energy entry point (vqemps_energy_noalloc).

It serves callers that must not allocate device memory while they run (a
simulator plugin inside a runtime that owns the device memory, an operator
under a fixed memory budget): all of its scratch lives in one static device
array. This file is collected last so that a run stopping at the first
failure has already run every other test; it also passes alone in a fresh
process. The checks: through the C ABI, two calls in a row give the energies and
per-term values of the existing batched entry point within the tolerance of the
other energy tests (1e-9 relative); further calls leave the device's free memory
unchanged (they allocate nothing); the caller's current device is kept; and
sizes beyond the limits are refused.
"""
import ctypes

import numpy as np
import pytest
import torch

from oracle import workloads as W

pytestmark = pytest.mark.gpu
RTOL = 1e-9


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_energy_matches_batched_entry_point_on_two_calls(cuda_device):
    import vqemps
    from vqemps import _lib
    lib = _lib.load()
    for spec, words, coeffs, thetas in (W.plain_12q(0)[:3] + (None,), W.batched_40q(0, batch=2)):
        eng = vqemps.Engine(0, 16)
        eng.set_spec(spec)
        ham = eng.set_hamiltonian(words, coeffs)
        if thetas is None:
            th0 = W.plain_12q(0)[3]
            thetas = np.stack([th0, th0 + 0.3])
        stream = torch.cuda.current_stream()
        for k in range(2):                                    # two calls in a row
            th = torch.tensor(thetas[k], dtype=torch.float64, device="cuda:0")
            e = torch.full((1,), -1.0, dtype=torch.float64, device="cuda:0")
            pt = torch.empty(len(words), dtype=torch.float64, device="cuda:0")
            st = torch.full((1,), 7, dtype=torch.int32, device="cuda:0")
            code = lib.vqemps_energy_noalloc(eng.ctx, ham.handle, _p(th), _p(e), _p(pt), _p(st),
                                             ctypes.c_void_p(stream.cuda_stream))
            assert code == _lib.OK, lib.vqemps_last_error(eng.ctx)
            ref_e, ref_pt = eng.energy(ham, th[None], per_term=True)
            torch.cuda.synchronize()
            assert int(st[0]) == 0
            assert abs(float(e[0]) - float(ref_e[0])) <= RTOL * max(1.0, abs(float(ref_e[0])))
            np.testing.assert_allclose(pt.cpu().numpy(), ref_pt[0].cpu().numpy(), rtol=0, atol=1e-11)
        eng.close()


def test_noalloc_calls_allocate_no_device_memory(cuda_device):
    """On a fresh engine, after its circuit and Pauli sum are loaded and one warm
    call (which loads the kernels), more calls leave cudaMemGetInfo's free
    memory exactly as it was; no batched call runs before, so no workspace of
    the engine could have been grown by them."""
    import vqemps
    from vqemps import _lib
    lib = _lib.load()
    spec, words, coeffs, thetas = W.batched_40q(0, batch=4)
    eng = vqemps.Engine(0, 16)
    eng.set_spec(spec)
    ham = eng.set_hamiltonian(words, coeffs)
    th = torch.tensor(thetas, dtype=torch.float64, device="cuda:0")
    e = torch.empty(4, dtype=torch.float64, device="cuda:0")
    st = torch.empty(4, dtype=torch.int32, device="cuda:0")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call(k):
        code = lib.vqemps_energy_noalloc(eng.ctx, ham.handle, _p(th[k]), _p(e[k:]), None, _p(st[k:]), stream)
        assert code == _lib.OK, lib.vqemps_last_error(eng.ctx)

    call(0)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for k in range(1, 4):
        call(k)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0
    assert (st == 0).all() and torch.isfinite(e).all()
    assert torch.cuda.current_device() == 0
    eng.close()


def test_noalloc_refuses_sizes_beyond_its_limits(cuda_device):
    import vqemps
    from vqemps import _lib
    from oracle.mps_oracle import hardware_efficient_spec
    lib = _lib.load()
    spec = hardware_efficient_spec(65, 1, ("ry",), "linear")
    eng = vqemps.Engine(0, 16)
    eng.set_spec(spec)
    ham = eng.set_hamiltonian(["Z" + "I" * 64], [1.0])
    th = torch.zeros(spec["count"], dtype=torch.float64, device="cuda:0")
    e = torch.empty(1, dtype=torch.float64, device="cuda:0")
    code = lib.vqemps_energy_noalloc(eng.ctx, ham.handle, _p(th), _p(e), None, None, None)
    assert code == _lib.INVALID
    assert b"exceed the limit of 64" in lib.vqemps_last_error(eng.ctx)
    eng.close()
