"""Geometry relaxation and atom-centre dynamics driven by the solver's forces.

Both drivers take an ``autograd.EnergyModel`` (or anything with ``evaluate(positions) ->
(E, F, _)``) and work in atomic units: positions in bohr, time in a.u. (1 fs = 41.341 a.u.),
masses in electron masses.

* ``fire``  -- FIRE relaxation (Bitzek, Koskinen, Gähler, Moseler, Gumbsch, PRL 97, 170201
  (2006)): damped MD with velocity mixing toward the force and an adaptive time step.
* ``velocity_verlet`` -- NVE velocity Verlet; returns the total-energy trajectory (drift).

Every force evaluation is one warm-started converged solve of the electronic problem (the state
carries over), which is what the benchmark workloads call "N imaginary-time iterations per step".
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List

import numpy as np

AMU = 1822.888486  # electron masses per unified atomic mass unit
MASS_AMU = {1: 1.008, 6: 12.011, 7: 14.007, 8: 15.999}
FS = 41.341374575751  # atomic time units per femtosecond


def masses_for(charges) -> np.ndarray:
    return np.array([MASS_AMU.get(int(round(z)), 2.0 * z) * AMU for z in charges])


@dataclass
class Trajectory:
    positions: List[np.ndarray] = field(default_factory=list)
    energies: List[float] = field(default_factory=list)
    fmax: List[float] = field(default_factory=list)
    kinetic: List[float] = field(default_factory=list)


def fire(model, x0, fmax: float = 1e-3, max_steps: int = 100, dt: float = 2.0, dt_max: float = 10.0,
         n_min: int = 5, f_inc: float = 1.1, f_dec: float = 0.5, alpha0: float = 0.1, f_alpha: float = 0.99,
         masses=None) -> Trajectory:
    """Relax nuclear positions x0 (n, 3) bohr until max |F| < fmax (Ha/bohr)."""
    x = np.array(x0, np.float64)
    m = np.ones(len(x)) if masses is None else np.asarray(masses, np.float64)
    v = np.zeros_like(x)
    alpha, since_neg = alpha0, 0
    traj = Trajectory()
    E, F, _ = model.evaluate(x)
    for _ in range(max_steps):
        f_max = float(np.abs(F).max())
        traj.positions.append(x.copy()); traj.energies.append(E); traj.fmax.append(f_max)
        if f_max < fmax:
            break
        power = float(np.sum(F * v))
        if power > 0:
            vn, fn = np.linalg.norm(v), np.linalg.norm(F)
            v = (1 - alpha) * v + alpha * vn * F / (fn + 1e-300)
            since_neg += 1
            if since_neg > n_min:
                dt = min(dt * f_inc, dt_max)
                alpha *= f_alpha
        else:
            v[:] = 0
            dt *= f_dec
            alpha, since_neg = alpha0, 0
        v += dt * F / m[:, None]
        x = x + dt * v
        E, F, _ = model.evaluate(x)
    return traj


def velocity_verlet(model, x0, v0, masses, dt: float, n_steps: int) -> Trajectory:
    """NVE velocity Verlet; traj.energies[i] + traj.kinetic[i] is the conserved total energy."""
    x = np.array(x0, np.float64)
    v = np.array(v0, np.float64)
    m = np.asarray(masses, np.float64)[:, None]
    E, F, _ = model.evaluate(x)
    traj = Trajectory()
    for _ in range(n_steps + 1):
        traj.positions.append(x.copy()); traj.energies.append(E)
        traj.kinetic.append(float(0.5 * np.sum(m * v * v))); traj.fmax.append(float(np.abs(F).max()))
        if len(traj.energies) > n_steps:
            break
        v_half = v + 0.5 * dt * F / m
        x = x + dt * v_half
        E, F, _ = model.evaluate(x)
        v = v_half + 0.5 * dt * F / m
    return traj
