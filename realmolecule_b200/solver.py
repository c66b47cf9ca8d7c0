"""Drop-in ``RealQMSolver`` for the Python host (cloud/solver.py:318-638).

Same constructor keys, same ``initialize()`` / ``run(total_steps, norm_interval,
poisson_interval, force_interval, report_interval)`` signature, same snapshot dicts and
public attributes (``E, E_T, E_eK, E_ee, E_KK, atom_pos, nuc_force, U, label``) as the
reference class; the solver step itself runs in librq on the GPU (CUDA graphs of whole
schedule periods), and only the reference's host-side logic (nuclear Euler move,
energy bookkeeping, reporting) stays in Python.

Extensions (optional config keys): ``flavor`` ("solver.py" default, "molecule.js",
"new") and ``precision`` ("mixed" default, "fp64" for the new flavour).
"""
from __future__ import annotations

import time
from typing import List, Optional

import numpy as np

from . import _lib as L
from .context import Context


class RealQMSolver:
    """GPU RealQM solver with the cloud/solver.py interface, backed by librq."""

    def __init__(self, config):
        self.NN = config["gridN"]
        self.S = self.NN + 1
        self.S3 = self.S ** 3
        self.screen = config["screen"]
        self.h = self.screen / self.NN
        self.h2 = self.h * self.h
        self.h3 = self.h ** 3
        self.N2 = self.NN // 2

        atoms = config["atoms"]
        self.nAtoms = len(atoms)
        self.Z_eff = np.array([a["Z"] for a in atoms], dtype=np.float32)
        self.atom_pos = np.array([[a["i"], a["j"], a.get("k", self.N2)] for a in atoms], dtype=np.float32)
        self.atom_rc = np.array([a.get("rc", 0) for a in atoms], dtype=np.float32)
        self.atom_el = [a.get("el", "") for a in atoms]
        self.active = self.Z_eff > 0
        self.nElec = int(self.active.sum())
        self._atom_rows = [dict(a) for a in atoms]

        self.flavor = config.get("flavor", "solver.py")
        ctx_opts = {k: config[k] for k in ("dv", "sigma", "mg_levels", "steps_per_frame") if k in config}
        self.ctx = Context(self.NN, self.screen, self._rows(), flavor=self.flavor,
                           precision=config.get("precision", "mixed"), **ctx_opts)
        self.dv = self.ctx.dv
        self.half_dv = 0.5 * self.dv
        self.dtv = self.dv * self.h2

        # dynamics parameters (cloud/solver.py:356-362)
        self.force_scale = config.get("forceScale", 1.0)
        self.damping = config.get("damping", 0.98)
        self.dt_nuc = config.get("dt_nuc", 0.8 if self.nElec <= 5 else 0.2 if self.nElec > 200 else 0.8)
        self.max_vel = 0.3 if self.nElec <= 5 else 0.03 if self.nElec > 200 else 0.1
        self.dynamics_enabled = config.get("dynamics", False)
        self._nProtein = config.get("nProtein", self.nAtoms)
        self._config_force_interval = config.get("force_interval", 500)
        self.nuc_vel = np.zeros((self.nAtoms, 3), dtype=np.float32)
        self.nuc_force = np.zeros((self.nAtoms, 3), dtype=np.float32)

        self.E_T = self.E_eK = self.E_ee = self.E_KK = self.E = 0.0
        self._atom_ref = {"H": -0.5, "O": -2.04, "C": -5.43, "N": -3.64}  # cloud/solver.py:396
        self.E_atoms_sum = sum(self._atom_ref.get(a.get("el", ""), 0) for a in atoms if a["Z"] > 0)
        self._initialized = False
        self._step = 0

    def _rows(self):
        rows = []
        for n, a in enumerate(self._atom_rows):
            r = dict(a)
            r["i"], r["j"], r["k"] = (float(x) for x in self.atom_pos[n])
            r["Z"] = float(self.Z_eff[n])
            r["rc"] = float(self.atom_rc[n])
            rows.append(r)
        return rows

    # -- state views (the reference exposes cupy arrays; here host copies) ------------------
    @property
    def U(self) -> np.ndarray:
        return self.ctx.download(psi=True, label=False)["psi"]

    @property
    def label(self) -> np.ndarray:
        return self.ctx.download(psi=False, label=True)["label"]

    # -- reference methods ------------------------------------------------------------------
    def initialize(self):
        """cloud/solver.py:402-419: trial state, normalise, 100 Poisson bootstrap steps."""
        self.ctx.initialize()
        self._initialized = True
        self._step = 0

    def _compute_energy(self):
        """cloud/solver.py:446-476 (FP64 sums on the GPU; E_KK with h^2 softening)."""
        e = self.ctx.energy()
        self.E_T, self.E_eK, self.E_ee, self.E_KK = (float(e[L.E_T]), float(e[L.E_EK]), float(e[L.E_EE]),
                                                     float(e[L.E_KK]))
        self.E = self.E_T + self.E_eK + self.E_ee + self.E_KK

    def _compute_forces(self):
        """cloud/solver.py:478-520: electronic HF forces on the atoms the reference batches
        (first nProtein, rounded up to its 32-atom batches), plus nuclear pair forces on the
        first nProtein atoms."""
        F = self.ctx.forces(L.FORCE_HF)
        nForce = self._nProtein
        end = min(self.nAtoms, ((nForce + 31) // 32) * 32) if nForce > 0 else 0
        self.nuc_force = np.zeros((self.nAtoms, 3), dtype=np.float32)
        self.nuc_force[:end] = F[:end].astype(np.float32)
        _, Fn = self.ctx.nuclear_terms()
        self.nuc_force[:nForce] += Fn[:nForce].astype(np.float32)

    def _move_nuclei(self):
        """cloud/solver.py:522-548: damped Euler on the first nProtein atoms, then K rebuild."""
        mass_map = {1: 1 * 1836, 2: 16 * 1836, 3: 14 * 1836, 4: 12 * 1836}
        for n in range(self._nProtein):
            z = int(self.Z_eff[n])
            if z <= 0:
                continue
            m = mass_map.get(z, 1836)
            for d in range(3):
                self.nuc_vel[n][d] += self.nuc_force[n][d] / m * self.dt_nuc * self.force_scale
                self.nuc_vel[n][d] *= self.damping
                self.nuc_vel[n][d] = np.clip(self.nuc_vel[n][d], -self.max_vel, self.max_vel)
                self.atom_pos[n][d] += self.nuc_vel[n][d] * self.dt_nuc / self.h
                self.atom_pos[n][d] = np.clip(self.atom_pos[n][d], 5, self.NN - 5)
        self.ctx.set_atoms(self._rows())

    def run(self, total_steps, norm_interval=20, poisson_interval=2, force_interval=None, report_interval=500):
        """cloud/solver.py:550-634.  Steps between events run as one librq call."""
        if force_interval is None:
            force_interval = self._config_force_interval
        if norm_interval != 20 or poisson_interval != 2:
            if (self.ctx.cfg.norm_interval, self.ctx.cfg.poisson_interval) != (norm_interval, poisson_interval):
                raise ValueError("norm_interval / poisson_interval are fixed when the context is created; "
                                 "pass them in the config")
        if not self._initialized:
            self.initialize()
        results: List[dict] = []
        t0 = time.time()
        step = 0
        while step < total_steps:
            nxt = total_steps
            for iv, on in ((force_interval, self.dynamics_enabled), (report_interval, True)):
                if on and iv:
                    nxt = min(nxt, (step // iv + 1) * iv)
            self.ctx.step(nxt - step)
            step = nxt
            if self.dynamics_enabled and force_interval and step % force_interval == 0:
                self._compute_forces()
                self._move_nuclei()
            if report_interval and step % report_interval == 0:
                self._compute_energy()
                elapsed = time.time() - t0
                ms_per_step = elapsed / step * 1000
                snap = {
                    "step": int(step), "E": float(self.E), "E_T": float(self.E_T), "E_eK": float(self.E_eK),
                    "E_ee": float(self.E_ee), "E_KK": float(self.E_KK), "E_bind": float(self.E - self.E_atoms_sum),
                    "ms_per_step": float(ms_per_step), "elapsed_sec": float(elapsed),
                    "nucPos": [[float(x) for x in row] for row in self.atom_pos],
                }
                if getattr(self, "_fold_atoms", None):
                    fa = self._fold_atoms
                    a, b, c = (self.atom_pos[fa[q]] * self.h for q in range(3))
                    ba, bc = a - b, c - b
                    mag = np.linalg.norm(ba) * np.linalg.norm(bc)
                    snap["fold_angle"] = float(np.degrees(np.arccos(np.clip(np.dot(ba, bc) / mag, -1, 1)))
                                               if mag > 0 else 0)
                results.append(snap)
        self.ctx.synchronize()
        return results

    def set_fold_atoms(self, indices):
        self._fold_atoms = indices
