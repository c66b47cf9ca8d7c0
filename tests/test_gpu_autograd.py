"""Differentiation and drivers on the GPU (new flavour, FP64 path): torch autograd of the
converged energy and of the energy after a fixed number of warm-started steps (the adjoint
through them, with the external potential and its gradient as CUDA tensors) against central
finite differences, FIRE relaxation of a stretched H2, and velocity-Verlet energy conservation."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def h2_model(R=1.6, NN=32, h=0.3, **kw):
    from realmolecule_b200.autograd import EnergyModel
    c = NN * h / 2
    pos = np.array([[c - R / 2, c, c], [c + R / 2, c + 0.003, c]])
    seeds = pos + np.array([[0.02, 0, 0], [-0.02, 0, 0]])
    return EnergyModel(NN, h, [1.0, 1.0], pos, seeds, **kw), pos


def test_autograd_positions_and_external_potential():
    from realmolecule_b200.autograd import energy
    model, pos = h2_model(tol=1e-12)
    S = model.NN + 1
    g = np.arange(S) * model.h
    X, Y, Zc = np.meshgrid(g, g, g, indexing="ij")
    bump = 0.05 * np.exp(-((X - pos[0, 0]) ** 2 + (Y - pos[0, 1] - 0.5) ** 2 + (Zc - pos[0, 2]) ** 2)).reshape(-1)
    R = torch.tensor(pos, dtype=torch.float64, requires_grad=True)
    v = torch.tensor(0.5 * bump, dtype=torch.float64, requires_grad=True)
    E = energy(R, model, v)
    E.backward()
    gR, gv = R.grad.numpy().copy(), v.grad.numpy().copy()
    d = 1e-3
    for a, ax in ((0, 0), (1, 1)):
        Es = []
        for s in (+1, -1):
            p2 = pos.copy()
            p2[a, ax] += s * d
            Es.append(model.evaluate(p2, 0.5 * bump)[0])
        assert abs((Es[0] - Es[1]) / (2 * d) - gR[a, ax]) < 1e-4
    # directional derivative along the bump itself: d/de E(v + e bump) = gv . bump
    Es = [model.evaluate(pos, (0.5 + s * 0.01) * bump)[0] for s in (+1, -1)]
    fd = (Es[0] - Es[1]) / 0.02
    assert abs(fd - float(gv @ bump)) < 1e-5 * max(1.0, abs(fd))


def test_fire_relaxes_h2():
    from realmolecule_b200.dynamics import fire
    model, pos = h2_model(R=2.0, tol=1e-9)
    tr = fire(model, pos, fmax=2e-3, max_steps=60)
    assert tr.fmax[-1] < tr.fmax[0] / 5
    assert tr.energies[-1] < tr.energies[0]


def test_velocity_verlet_energy_drift():
    from realmolecule_b200.dynamics import masses_for, velocity_verlet, FS
    model, pos = h2_model(R=1.5, tol=1e-11)
    # H2 vibrates with a ~8 fs period: 0.1 fs keeps the Verlet energy error (O(dt^2)) small
    tr = velocity_verlet(model, pos, np.zeros_like(pos), masses_for([1, 1]), dt=0.1 * FS, n_steps=10)
    tot = np.array(tr.energies) + np.array(tr.kinetic)
    assert np.max(np.abs(tot - tot[0])) < 1e-4
    assert tr.kinetic[-1] > 1e-5  # the stretched bond did start to move


def test_autograd_warm_started_energy_on_the_device():
    """tol=None: every evaluation runs 48 warm-started steps and its gradient is the adjoint through
    them.  v and dE/dv stay CUDA tensors.  Each evaluation here restarts from one saved state, so
    E(R, v) is one function; bar 1e-4 Ha/bohr (positions), 1e-6 relative (along v)."""
    from realmolecule_b200.autograd import energy
    model, pos = h2_model(tol=None, warm_steps=48, label_until=200)
    model.ctx.step(200)  # not converged: the reverse sweep carries a real correction
    st = model.ctx.download(psi=True, label=False, P=True)
    S = model.NN + 1
    g = np.arange(S) * model.h
    X, Y, Zc = np.meshgrid(g, g, g, indexing="ij")
    bump = 0.05 * np.exp(-((X - pos[0, 0]) ** 2 + (Y - pos[0, 1] - 0.5) ** 2 + (Zc - pos[0, 2]) ** 2)).reshape(-1)

    def E_at(p, v):
        model.ctx.upload(psi=st["psi"], P=st["P"])
        return model.evaluate(p, v)[0]

    model.ctx.upload(psi=st["psi"], P=st["P"])
    R = torch.tensor(pos, dtype=torch.float64, requires_grad=True)
    v = torch.tensor(0.5 * bump, dtype=torch.float64, device="cuda", requires_grad=True)
    E = energy(R, model, v)
    E.backward()
    assert v.grad.is_cuda
    gR, gv = R.grad.numpy().copy(), v.grad.cpu().numpy()
    d = 1e-3
    for a, ax in ((0, 0), (1, 1)):
        Es = []
        for s in (+1, -1):
            p2 = pos.copy()
            p2[a, ax] += s * d
            Es.append(E_at(p2, 0.5 * bump))
        assert abs((Es[0] - Es[1]) / (2 * d) - gR[a, ax]) < 1e-4
    Es = [E_at(pos, (0.5 + s * 0.01) * bump) for s in (+1, -1)]
    fd = (Es[0] - Es[1]) / 0.02
    assert abs(fd - float(gv @ bump)) < 1e-6 * max(1.0, abs(fd))
