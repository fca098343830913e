"""MPSEnergy's choice between the adjoint sweep and the energy-only path, on a
stand-in engine (host logic only; the GPU tests cover the kernels)."""
import torch

from vqemps.reverse import MPSEnergy, mps_energy


class FakeEngine:
    device = torch.device("cpu")

    def __init__(self):
        self.calls = []

    def energy(self, ham, th):
        self.calls.append("energy")
        return (th ** 2).sum(1)

    def energy_grad(self, ham, th):
        self.calls.append("energy_grad")
        return (th ** 2).sum(1), 2 * th


def test_gradient_path_only_when_autograd_needs_it():
    eng = FakeEngine()
    x = torch.tensor([[1.0, 2.0], [0.5, -1.0]], dtype=torch.float64, requires_grad=True)
    e = MPSEnergy.apply(x, eng, None)
    e.sum().backward()
    assert eng.calls == ["energy_grad"]
    assert torch.equal(x.grad, 2 * x.detach())
    with torch.no_grad():
        e2 = mps_energy(x, eng, None)
    assert eng.calls[-1] == "energy" and torch.equal(e2, e.detach())
    mps_energy(x.detach(), eng, None)
    assert eng.calls[-1] == "energy"
    y = torch.tensor([3.0, -1.0], dtype=torch.float64, requires_grad=True)
    ey = mps_energy(y, eng, None)
    assert ey.dim() == 0
    ey.backward()
    assert eng.calls[-1] == "energy_grad" and torch.equal(y.grad, 2 * y.detach())
