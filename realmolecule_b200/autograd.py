"""Differentiable energy of the new flavour, for PyTorch.

``EnergyModel`` owns one new-flavour context (Gaussian nuclei, multigrid Hartree, FP64 domain
sums) and evaluates the energy E(R, v) for nuclear positions R (bohr, box frame: x = i*h) and an
optional external potential v on the grid.  Every evaluation warm-starts from the previous
state (labels frozen after the first ``label_until`` steps) and either

* solves to a tolerance (``tol`` given): E is the converged energy; or
* runs exactly ``warm_steps`` imaginary-time steps (``tol=None``, the geometry workloads): E is
  the energy those steps reach.

Its gradients come from librq's adjoint (``rq_adjoint``): the steps of each evaluation are
recorded (``rq_set_adjoint_window``) and a reverse sweep through them -- the update, the
per-domain normalisation and the multigrid V-cycle transposed -- gives the exact dE/dR and
dE/dv of the energy actually reached, converged or not.  For a solve to a tolerance the
recorded window is empty and the gradient is the Hellmann-Feynman one, exact at convergence.

``RealQMEnergy`` wraps an EnergyModel as a ``torch.autograd.Function``.  An external potential
given as a float64 CUDA tensor is read on the device and its gradient written on the device.
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
                 check_interval: int = 100, warm_steps: int = 0, adjoint: bool = True, cold: bool = False,
                 **opts):
        """tol None: each evaluation runs exactly ``warm_steps`` imaginary-time steps from the previous
        state (the fixed warm-started iterations of the geometry workloads) instead of a solve, and
        those steps are recorded for the adjoint.  adjoint False: no recording; the gradient is the
        Hellmann-Feynman one (exact only at convergence), for comparison.  cold True (with tol None):
        every evaluation starts from the initial state (nearest-seed labels, held fixed), so E is a
        function of the positions alone -- E_N(R) -- and the adjoint force is its exact gradient."""
        self.NN, self.h = int(NN), float(h)
        self.S3 = (self.NN + 1) ** 3
        self.charges = np.asarray(charges, np.float64)
        self.n_nuc = len(self.charges)
        self.seeds = np.asarray(seeds, np.float64)
        self.tol, self.max_steps, self.check = tol, max_steps, check_interval
        self.warm_steps = warm_steps
        rows = self._rows(np.asarray(positions, np.float64))
        self.cold = bool(cold) and tol is None
        opts.setdefault("label_until", 1 if self.cold else 400)
        self.ctx = Context(self.NN, self.NN * self.h, rows, flavor="new", precision=precision, **opts)
        self.ctx.initialize()
        if not self.cold:
            self.ctx.step(opts["label_until"])  # let the level set settle, then labels stay fixed
        if adjoint and tol is None and warm_steps > 0:
            self.ctx.set_adjoint_window(warm_steps)
        self._has_v = False
        self.last = None

    def _rows(self, pos: np.ndarray):
        rows = [{"i": p[0] / self.h, "j": p[1] / self.h, "k": p[2] / self.h, "Z": 0.0, "Z_nuc": float(z)}
                for p, z in zip(pos, self.charges)]
        rows += [{"i": s[0] / self.h, "j": s[1] / self.h, "k": s[2] / self.h, "Z": 1.0, "Z_nuc": 0.0}
                 for s in self.seeds]
        return rows

    def evaluate(self, positions: np.ndarray, v=None, dE_dv=None):
        """Energy and total forces on the nuclei (n_nuc x 3) for positions R and external potential v
        (S^3 values: numpy array or float64 torch tensor, None for none).  With dE_dv (True, or a
        float64 tensor of S^3 values to fill) also returns dE/dv, else None."""
        positions = np.asarray(positions, np.float64).reshape(self.n_nuc, 3)
        self.ctx.set_atoms(self._rows(positions))
        if v is not None or self._has_v:
            self.ctx.set_external_potential(v)
            self._has_v = v is not None
        if self.tol is None:
            if self.cold:
                self.ctx.initialize()  # the state every evaluation starts from (independent of R)
            self.ctx.step(self.warm_steps)
            steps, E = self.warm_steps, float(self.ctx.energy()[L.E_TOTAL])
        else:
            steps, E = self.ctx.solve(self.tol, self.max_steps, self.check)
        Fe, g = self.ctx.adjoint(forces=True, potential=dE_dv if dE_dv is not None else False)
        _, Fn = self.ctx.nuclear_terms()
        F = Fe[: self.n_nuc] + Fn[: self.n_nuc]
        self.last = {"E": E, "F": F, "steps": steps}
        return E, F, g


class RealQMEnergy(torch.autograd.Function):
    """E = RealQMEnergy.apply(positions, v_ext, model): positions (n_nuc, 3) float64 bohr,
    v_ext (S^3,) float64 (host or CUDA) or an empty tensor for none."""

    @staticmethod
    def forward(ctx, positions, v_ext, model: EnergyModel):
        has_v = v_ext.numel() > 0
        v = v_ext.detach().contiguous() if has_v else None
        dv = torch.empty(model.S3, dtype=torch.float64, device=v_ext.device) if has_v else None
        if has_v and v.is_cuda:
            torch.cuda.synchronize(v.device)  # librq reads v on its own stream
        E, F, _ = model.evaluate(positions.detach().cpu().numpy(), v, dE_dv=dv)
        ctx.save_for_backward(torch.from_numpy(-F).to(positions.device), dv if has_v else v_ext.new_zeros(0))
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
