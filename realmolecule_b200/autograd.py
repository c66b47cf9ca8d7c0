"""Differentiable converged energy of the new flavour, for PyTorch.

``EnergyModel`` owns one new-flavour context (Gaussian nuclei, multigrid Hartree, FP64 domain
sums) and evaluates the converged energy E(R, v) for nuclear positions R (bohr, box frame:
x = i*h) and an optional external potential v on the grid.  ``RealQMEnergy`` wraps it as a
``torch.autograd.Function``:

* dE/dR  = -(F_electronic + F_nuclear), with F_electronic the gradient kernel of librq
  (``rq_forces(RQ_FORCE_ADJOINT)``).  At a converged state with the domain labels held fixed the
  electronic energy is stationary in psi under the per-domain norm constraints, so the adjoint
  of the psi equations vanishes and this is the exact derivative of the discrete energy
  (checked against central finite differences in the tests);
* dE/dv  = -h^3 rho  (v enters as K + v, E_eK = -h^3 sum (K + v) rho).

Every evaluation warm-starts from the previous state: labels are frozen after the first solve.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib as L
from .context import Context


class EnergyModel:
    def __init__(self, NN: int, h: float, charges: Sequence[float], positions: np.ndarray,
                 seeds: np.ndarray, precision: str = "fp64", tol: Optional[float] = 1e-10, max_steps: int = 50000,
                 check_interval: int = 100, warm_steps: int = 0, want_rho: bool = True, **opts):
        """tol None: each evaluation runs exactly ``warm_steps`` imaginary-time steps from the previous
        state (the fixed warm-started iterations of the geometry workloads) instead of a solve.
        want_rho False: evaluate returns None for h^3 rho (no density download)."""
        self.NN, self.h = int(NN), float(h)
        self.want_rho = want_rho
        self.charges = np.asarray(charges, np.float64)
        self.n_nuc = len(self.charges)
        self.seeds = np.asarray(seeds, np.float64)
        self.tol, self.max_steps, self.check = tol, max_steps, check_interval
        self.warm_steps = warm_steps
        rows = self._rows(np.asarray(positions, np.float64))
        opts.setdefault("label_until", 400)
        self.ctx = Context(self.NN, self.NN * self.h, rows, flavor="new", precision=precision, **opts)
        self.ctx.initialize()
        self.ctx.step(opts["label_until"])  # let the level set settle, then labels stay fixed
        self._v = None
        self.last = None

    def _rows(self, pos: np.ndarray):
        rows = [{"i": p[0] / self.h, "j": p[1] / self.h, "k": p[2] / self.h, "Z": 0.0, "Z_nuc": float(z)}
                for p, z in zip(pos, self.charges)]
        rows += [{"i": s[0] / self.h, "j": s[1] / self.h, "k": s[2] / self.h, "Z": 1.0, "Z_nuc": 0.0}
                 for s in self.seeds]
        return rows

    def evaluate(self, positions: np.ndarray, v: Optional[np.ndarray] = None):
        """Converged energy, total forces on the nuclei (n_nuc x 3) and h^3 rho for positions R
        (h^3 rho is None when the model was built with want_rho=False and no v is given)."""
        positions = np.asarray(positions, np.float64).reshape(self.n_nuc, 3)
        self.ctx.set_atoms(self._rows(positions))
        if v is not None or self._v is not None:
            self.ctx.set_external_potential(v)
            self._v = v
        if self.warm_steps:
            self.ctx.step(self.warm_steps)
        if self.tol is None:
            steps, E = self.warm_steps, float(self.ctx.energy()[L.E_TOTAL])
        else:
            steps, E = self.ctx.solve(self.tol, self.max_steps, self.check)
        Fe = self.ctx.forces(L.FORCE_ADJOINT)[: self.n_nuc]
        _, Fn = self.ctx.nuclear_terms()
        F = Fe + Fn[: self.n_nuc]
        rho_h3 = None
        if self.want_rho or v is not None:  # dE/dv = -h^3 rho needs the density whenever v is given
            psi = self.ctx.download(psi=True, label=False)["psi"].astype(np.float64)
            rho_h3 = psi * psi * self.h ** 3
        self.last = {"E": E, "F": F, "steps": steps}
        return E, F, rho_h3


class RealQMEnergy(torch.autograd.Function):
    """E = RealQMEnergy.apply(positions, v_ext, model): positions (n_nuc, 3) float64 bohr,
    v_ext (S^3,) float64 or an empty tensor for none."""

    @staticmethod
    def forward(ctx, positions, v_ext, model: EnergyModel):
        v = v_ext.detach().cpu().numpy() if v_ext.numel() else None
        E, F, rho_h3 = model.evaluate(positions.detach().cpu().numpy(), v)
        ctx.save_for_backward(torch.from_numpy(-F).to(positions.device),
                              torch.from_numpy(-rho_h3).to(v_ext.device) if v_ext.numel() else v_ext.new_zeros(0))
        return torch.tensor(E, dtype=torch.float64, device=positions.device)

    @staticmethod
    def backward(ctx, grad_E):
        dE_dR, dE_dv = ctx.saved_tensors
        g_pos = grad_E * dE_dR if ctx.needs_input_grad[0] else None
        g_v = grad_E * dE_dv if (ctx.needs_input_grad[1] and dE_dv.numel()) else None
        return g_pos, g_v, None


def energy(positions: torch.Tensor, model: EnergyModel, v_ext: Optional[torch.Tensor] = None) -> torch.Tensor:
    if v_ext is None:
        v_ext = torch.zeros(0, dtype=torch.float64, device=positions.device)
    return RealQMEnergy.apply(positions, v_ext, model)
