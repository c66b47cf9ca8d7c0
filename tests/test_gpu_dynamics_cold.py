"""Velocity Verlet on E_N(R): the energy N imaginary-time steps reach from the same initial state
(cold start, labels fixed by the domain seeds), so E_N is a function of the positions alone.

The adjoint force is the exact gradient of E_N, so the total energy E_N + kinetic is conserved up
to the integrator's O(dt^2) error; the Hellmann-Feynman force of the unconverged state is not a
gradient of E_N, and the total energy drifts.  One water on 64^3 (h = 0.25 bohr), N = 80, FP64,
20 steps of 1 a.u. from rest.  Bar: the adjoint run's largest total-energy excursion is below a
fifth of the Hellmann-Feynman run's and below 1e-4 Ha.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_adjoint_forces_conserve_the_cold_start_energy():
    from realmolecule_b200 import configs as C
    from realmolecule_b200.autograd import EnergyModel
    from realmolecule_b200.dynamics import masses_for, velocity_verlet
    g = C.h2o64()
    off = (g.NN // 2) * g.h
    x0 = g.xyz + off
    exc = {}
    for adjoint in (True, False):
        model = EnergyModel(g.NN, g.h, g.charges, x0, g.seeds + off, precision="fp64", tol=None, warm_steps=80,
                            adjoint=adjoint, cold=True)
        tr = velocity_verlet(model, x0, np.zeros_like(x0), masses_for(g.charges), dt=1.0, n_steps=20)
        Et = np.array(tr.energies) + np.array(tr.kinetic)
        exc[adjoint] = float(np.abs(Et - Et[0]).max())
        model.ctx.close()
    assert exc[True] < 0.2 * exc[False] and exc[True] < 1e-4, exc
