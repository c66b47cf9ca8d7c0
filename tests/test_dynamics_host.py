"""Host logic of the autograd wrapper and the FIRE / velocity-Verlet drivers, on an analytic
model (no GPU): harmonic wells whose energy and forces are known in closed form."""
import numpy as np
import torch

from realmolecule_b200.autograd import RealQMEnergy
from realmolecule_b200.dynamics import fire, velocity_verlet


class Harmonic:
    """E = sum_a k/2 |x_a - c_a|^2 + sum_x v(x) w(x): forces -k (x - c); dE/dv = w.  The same
    interface as autograd.EnergyModel: evaluate(x, v, dE_dv) fills a given dE_dv tensor."""

    def __init__(self, centres, k=0.3, w=None):
        self.c = np.asarray(centres, float)
        self.k = k
        self.w = w
        self.S3 = len(w) if w is not None else 0
        self.calls = 0

    def evaluate(self, x, v=None, dE_dv=None):
        self.calls += 1
        x = np.asarray(x, float).reshape(self.c.shape)
        E = 0.5 * self.k * np.sum((x - self.c) ** 2)
        if v is not None:
            E += float(np.dot(np.asarray(v.cpu() if hasattr(v, "cpu") else v), self.w))
        if dE_dv is not None:
            dE_dv.copy_(torch.from_numpy(self.w))
        return E, -self.k * (x - self.c), dE_dv


def test_autograd_function_routes_gradients():
    m = Harmonic([[0, 0, 0], [1.0, 0, 0]], w=np.linspace(0, 1, 5))
    R = torch.tensor([[0.1, 0.2, 0.0], [1.3, 0.0, -0.1]], dtype=torch.float64, requires_grad=True)
    v = torch.linspace(-1, 1, 5, dtype=torch.float64, requires_grad=True)
    E = RealQMEnergy.apply(R, v, m)
    E.backward()
    np.testing.assert_allclose(R.grad.numpy(), m.k * (R.detach().numpy() - m.c))
    np.testing.assert_allclose(v.grad.numpy(), m.w)


def test_fire_relaxes_to_the_minimum():
    m = Harmonic([[0, 0, 0], [1.5, 0.2, -0.3]])
    tr = fire(m, [[0.5, -0.4, 0.2], [2.2, 0.5, 0.0]], fmax=1e-6, max_steps=500)
    assert tr.fmax[-1] < 1e-6
    np.testing.assert_allclose(tr.positions[-1], m.c, atol=1e-4)
    assert tr.energies[-1] < tr.energies[0]


def test_velocity_verlet_conserves_energy():
    m = Harmonic([[0, 0, 0]], k=1.0)
    tr = velocity_verlet(m, [[1.0, 0, 0]], [[0, 0.5, 0]], masses=[1.0], dt=0.01, n_steps=2000)
    tot = np.array(tr.energies) + np.array(tr.kinetic)
    assert np.max(np.abs(tot - tot[0])) < 1e-4
