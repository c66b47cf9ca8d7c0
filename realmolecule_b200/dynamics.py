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


def geometry_model(g, precision: str = "mixed", iters: int = 200, label_until: int = 400, adjoint: bool = True):
    """An EnergyModel for a configs.Geometry in the workloads' mode: each evaluation runs `iters`
    warm-started imaginary-time steps (no solve to a tolerance) and its forces are the exact
    gradient of the energy those steps reach (the adjoint through them; adjoint False: the
    Hellmann-Feynman force of the state reached)."""
    from .autograd import EnergyModel
    off = (g.NN // 2) * g.h  # geometries are centred on the centroid; the model uses the box frame
    return EnergyModel(g.NN, g.h, g.charges, g.xyz + off, g.seeds + off, precision=precision, tol=None,
                       warm_steps=iters, label_until=label_until, adjoint=adjoint), g.charges, off


def _main(argv=None):
    """Run the geometry workloads of the benchmark configurations on cuda:0.

    python -m realmolecule_b200.dynamics --workload water100 [--steps 100] [--iters 200]
        FIRE relaxation of 100 waters (192^3), each step warm-started with `iters` iterations.
    python -m realmolecule_b200.dynamics --workload water1000 [--steps 200] [--iters 50] [--dt-fs 0.5]
        velocity Verlet of 1000 waters (320^3); prints the total-energy drift.
    Prints one JSON line (per-step wall times, energies, fmax / drift)."""
    import argparse
    import json
    import time

    from . import _lib as L, configs
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--workload", default="water100", choices=["water100", "water1000"])
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--iters", type=int, default=None)
    ap.add_argument("--dt-fs", type=float, default=0.5)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--forces", default="adjoint", choices=["adjoint", "hf"],
                    help="adjoint: exact gradient of the energy reached; hf: Hellmann-Feynman of the state")
    ap.add_argument("--preconverge", type=int, default=None,
                    help="imaginary-time steps before the first geometry step (default 2000 / 3000)")
    a = ap.parse_args(argv)
    g = configs.water100() if a.workload == "water100" else configs.water1000()
    iters = a.iters or (200 if a.workload == "water100" else 50)
    t0 = time.perf_counter()
    model, Z, off = geometry_model(g, a.precision, iters, adjoint=a.forces == "adjoint")
    pre = a.preconverge if a.preconverge is not None else (2000 if a.workload == "water100" else 3000)
    model.ctx.step(pre)  # converge the electrons at the start geometry
    model.ctx.synchronize()
    t_init = time.perf_counter() - t0
    # one evaluation split into its parts (synchronised wall clock; per kernel class, CUDA events)
    parts, kernels = {}, {}
    for name, fn in (("set_atoms_ms", lambda: model.ctx.set_atoms(model._rows(g.xyz + off))),
                     ("iters_ms", lambda: model.ctx.step(iters)), ("energy_ms", lambda: model.ctx.energy()),
                     ("forces_ms", lambda: model.ctx.forces(L.FORCE_ADJOINT))):
        model.ctx.profile_begin()
        t1 = time.perf_counter(); fn(); model.ctx.synchronize(); parts[name] = (time.perf_counter() - t1) * 1e3
        kernels[name] = {k: round(v["ms"], 3) for k, v in model.ctx.profile_end().items()}
    m = masses_for(Z)
    t0 = time.perf_counter()
    if a.workload == "water100":
        tr = fire(model, g.xyz + off, max_steps=a.steps or 100, masses=m)
        out = {"fmax_first": tr.fmax[0], "fmax_last": tr.fmax[-1], "E_first": tr.energies[0], "E_last": tr.energies[-1]}
    else:
        n = a.steps or 200
        tr = velocity_verlet(model, g.xyz + off, np.zeros_like(g.xyz), m, a.dt_fs * FS, n)
        Et = np.array(tr.energies) + np.array(tr.kinetic)
        out = {"E_total_first": float(Et[0]), "E_total_last": float(Et[-1]),
               "drift_Ha": float(Et[-1] - Et[0]), "max_excursion_Ha": float(np.abs(Et - Et[0]).max())}
    dt = time.perf_counter() - t0
    nstep = len(tr.energies)
    print(json.dumps({"workload": a.workload, "forces": a.forces, "grid": f"{g.NN}^3", "nuclei": len(Z),
                      "domains": len(g.seeds),
                      "iters_per_step": iters, "preconverge_steps": pre, "steps": nstep, "init_s": t_init, "s": dt,
                      "evaluation_parts": parts, "evaluation_kernel_ms": kernels,
                      "ms_per_geometry_step": dt / max(1, nstep) * 1e3, **out}), flush=True)


if __name__ == "__main__":
    _main()
