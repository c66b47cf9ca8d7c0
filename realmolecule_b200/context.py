"""Thin object wrapper over one librq context (include/rq.h).

``Context`` owns an ``rq_ctx``: it creates it from a flavour, grid and atom list, and
exposes the step, energies, forces and state transfer with numpy arrays on the host.
Device pointers of the live fields are available through ``info()`` for zero-copy use
(e.g. wrapping them as torch tensors).
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Optional, Sequence

import numpy as np

from . import _lib as L

FLAVORS = {"molecule.js": L.FLAVOR_MOLECULE_JS, "molecule": L.FLAVOR_MOLECULE_JS, "solver.py": L.FLAVOR_SOLVER_PY,
           "solverpy": L.FLAVOR_SOLVER_PY, "new": L.FLAVOR_NEW}
PRECISIONS = {"mixed": L.PREC_MIXED, "fp32": L.PREC_MIXED, "fp64": L.PREC_FP64}


def make_atoms(rows: Iterable[dict], default_k: Optional[float] = None):
    """Reference atom dicts ({i, j, k, Z, rc, Z_nuc, initZeff, initRcut}) -> ctypes array."""
    rows = list(rows)
    arr = (L.Atom * len(rows))()
    for n, a in enumerate(rows):
        arr[n].i = float(a["i"])
        arr[n].j = float(a["j"])
        arr[n].k = float(a.get("k", default_k if default_k is not None else 0.0))
        arr[n].Z = float(a.get("Z", 0.0))
        arr[n].Z_nuc = float(a["Z_nuc"]) if a.get("Z_nuc") is not None else float(a.get("Z", 0.0))
        arr[n].rc = float(a.get("rc", 0.0) or 0.0)
        arr[n].init_zeff = float(a.get("initZeff", 0.0) or 0.0)
        arr[n].init_rcut = float(a.get("initRcut", 0.0) or 0.0)
    return arr


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.flags.c_contiguous
    return a.ctypes.data


class Context:
    """One solver grid on the current CUDA device."""

    def __init__(self, NN: int, screen: float, atoms: Sequence[dict], flavor: str = "solver.py",
                 precision: str = "mixed", **opts):
        self.lib = L.load()
        cfg = L.Config()
        cfg.NN = int(NN)
        cfg.screen = float(screen)
        cfg.flavor = FLAVORS[flavor] if isinstance(flavor, str) else int(flavor)
        cfg.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        for k, v in opts.items():
            if v is None:
                continue
            if not hasattr(cfg, k):
                raise TypeError(f"unknown option {k}")
            setattr(cfg, k, v)
        self.cfg = cfg
        self._atoms = make_atoms(atoms, default_k=NN // 2)
        self.n_atoms = len(self._atoms)
        h = C.c_void_p()
        st = self.lib.rq_create(C.byref(cfg), self._atoms, self.n_atoms, C.byref(h))
        L.check(st, "rq_create")
        self.ctx = h
        inf = self.info()
        self.S, self.NN, self.S3 = inf.S, inf.NN, inf.S3
        self.h, self.dv, self.dt = inf.h, inf.dv, inf.dt
        self.fp64 = inf.precision == L.PREC_FP64

    # -- lifecycle ------------------------------------------------------------------------
    def close(self):
        if getattr(self, "ctx", None):
            self.lib.rq_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st, where):
        return L.check(st, where, self.ctx)

    def info(self) -> L.Info:
        inf = L.Info()
        self._chk(self.lib.rq_get_info(self.ctx, C.byref(inf)), "rq_get_info")
        return inf

    def set_stream(self, stream_handle: int | None):
        self._chk(self.lib.rq_set_stream(self.ctx, stream_handle), "rq_set_stream")

    # -- solver ---------------------------------------------------------------------------
    def initialize(self):
        self._chk(self.lib.rq_initialize(self.ctx), "rq_initialize")

    def step(self, n: int = 1):
        self._chk(self.lib.rq_step(self.ctx, int(n)), "rq_step")

    def synchronize(self):
        self._chk(self.lib.rq_synchronize(self.ctx), "rq_synchronize")

    def energy(self, per_domain: bool = False):
        out = np.zeros(L.ENERGY_LEN, np.float64)
        pd = np.zeros((self.n_atoms, L.DOMAIN_LEN), np.float64) if per_domain else None
        self._chk(self.lib.rq_energy(self.ctx, _ptr(out), _ptr(pd)), "rq_energy")
        return (out, pd) if per_domain else out

    def forces(self, method: int = L.FORCE_HF) -> np.ndarray:
        F = np.zeros((self.n_atoms, 3), np.float64)
        self._chk(self.lib.rq_forces(self.ctx, int(method), _ptr(F)), "rq_forces")
        return F

    def nuclear_terms(self):
        e = C.c_double()
        F = np.zeros((self.n_atoms, 3), np.float64)
        self._chk(self.lib.rq_nuclear_terms(self.ctx, C.byref(e), _ptr(F)), "rq_nuclear_terms")
        return e.value, F

    def set_atoms(self, atoms: Sequence[dict]):
        arr = make_atoms(atoms, default_k=self.NN // 2)
        self._chk(self.lib.rq_set_atoms(self.ctx, arr, len(arr)), "rq_set_atoms")
        self._atoms = arr

    def set_init_positions(self, init_pos):
        """molecule.js window.USER_INIT_POS: per entry an (i, j) grid position for the next
        initialisation's trial psi and labels, or None (the entry's own position); K is rebuilt at
        the true positions.  An empty list clears."""
        n = len(init_pos)
        pos = np.zeros(2 * n, np.float64)
        has = np.zeros(n, np.int32)
        for q, p in enumerate(init_pos):
            if p is not None:
                pos[2 * q], pos[2 * q + 1], has[q] = float(p[0]), float(p[1]), 1
        self._chk(self.lib.rq_set_init_positions(self.ctx, _ptr(pos), _ptr(has), n), "rq_set_init_positions")

    def set_freeze_boundary(self, on: bool):
        """molecule.js flavour: window.FREEZE_BOUNDARY -- frames skip the level-set passes while on."""
        self._chk(self.lib.rq_set_freeze_boundary(self.ctx, 1 if on else 0), "rq_set_freeze_boundary")

    def restart(self):
        """molecule.js flavour: the classical-MD backbone's full restart at the current positions
        (K, trial psi, labels from scratch, P cleared; W and Pother kept)."""
        self._chk(self.lib.rq_restart(self.ctx), "rq_restart")

    def set_locked_groups(self, groups):
        """molecule.js flavour: window.USER_LOCKED_GROUPS (molecule.js:490-503), a list of label
        lists; a boundary between two labels of one group does not move.  [] removes them."""
        groups = [list(map(int, g)) for g in (groups or [])]
        offsets = np.zeros(len(groups) + 1, np.int32)
        offsets[1:] = np.cumsum([len(g) for g in groups], dtype=np.int64)
        members = np.asarray([m for g in groups for m in g] or [0], np.int32)
        self._chk(self.lib.rq_set_locked_groups(self.ctx, len(groups), _ptr(offsets), _ptr(members)),
                  "rq_set_locked_groups")

    def set_splits(self, splits):
        """molecule.js flavour: the shell split of every entry (USER_SPLIT_TYPE / _IDX / _AXIS / _ROT,
        molecule.js:27-32) as dicts {type: 'hemi'|'third'|2|3, idx, axis, rot} (None or {} = whole
        sphere); set before initialize().  None removes them."""
        if not splits:
            self._chk(self.lib.rq_set_splits(self.ctx, None), "rq_set_splits")
            return
        arr = (L.Split * len(self._atoms))()
        codes = {"sphere": 0, "hemi": 2, "third": 3, "tetra": 4}
        for n, sp in enumerate(splits):
            if not sp:
                continue
            t = sp.get("type", 0)
            arr[n].type = codes.get(t, 0) if isinstance(t, str) else int(t or 0)
            arr[n].idx = int(sp.get("idx", 0))
            arr[n].axis[:] = [float(v) for v in (sp.get("axis") or (0.0, 0.0, 1.0))]
            arr[n].rot = float(sp.get("rot", 0.0))
        self._chk(self.lib.rq_set_splits(self.ctx, arr), "rq_set_splits")

    def set_external_potential(self, v):
        """Add an external potential v (S^3 values, Ha) to K (new flavour); None removes it.  A
        contiguous float64 torch tensor on this GPU is read in place (no host round trip)."""
        if v is not None and hasattr(v, "data_ptr"):
            assert v.dtype.itemsize == 8 and v.is_contiguous() and v.numel() == self.S3
            self._chk(self.lib.rq_set_external_potential(self.ctx, v.data_ptr()), "rq_set_external_potential")
            return
        arr = None if v is None else np.ascontiguousarray(np.asarray(v, np.float64).reshape(-1))
        self._chk(self.lib.rq_set_external_potential(self.ctx, _ptr(arr)), "rq_set_external_potential")

    def extract(self, slice_k: int | None = None) -> np.ndarray:
        """molecule.js flavour: the page's slice buffer (3 S^2 + 2 S floats) at k = slice_k (N2)."""
        k = self.NN // 2 if slice_k is None else int(slice_k)
        out = np.empty(3 * self.S * self.S + 2 * self.S, np.float32)
        self._chk(self.lib.rq_extract(self.ctx, k, out.ctypes.data), "rq_extract")
        return out

    def promote(self):
        """New flavour: continue in FP64 from the current mixed-precision state (rq_promote)."""
        self._chk(self.lib.rq_promote(self.ctx), "rq_promote")
        self.fp64 = True

    def set_adjoint_window(self, steps: int):
        """New flavour: record the state of every following step, keeping the last `steps`, so that
        ``adjoint`` can run the reverse sweep through them (rq_set_adjoint_window; 0 = off)."""
        self._chk(self.lib.rq_set_adjoint_window(self.ctx, int(steps)), "rq_set_adjoint_window")

    def adjoint(self, forces: bool = True, potential=False):
        """Exact gradient of the energy readout through the recorded steps (rq_adjoint): returns
        (F, dE_dv) -- F = -dE/dR per entry (n_atoms x 3, electronic part) and dE/dv on the grid
        (S^3 doubles) -- each None unless asked for.  `potential` may be a contiguous float64 torch
        tensor of S^3 values (on this GPU or the host), which is filled in place and returned."""
        F = np.zeros((self.n_atoms, 3), np.float64) if forces else None
        if hasattr(potential, "data_ptr"):
            assert potential.dtype.itemsize == 8 and potential.is_contiguous() and potential.numel() == self.S3
            g, gp = potential, potential.data_ptr()
        else:
            g = np.zeros(self.S3, np.float64) if potential else None
            gp = _ptr(g)
        self._chk(self.lib.rq_adjoint(self.ctx, _ptr(F), gp), "rq_adjoint")
        return F, g

    def solve(self, tol_dE: float, max_steps: int, check_interval: int = 100):
        taken = C.c_int32()
        e = C.c_double()
        self._chk(self.lib.rq_solve(self.ctx, float(tol_dE), int(max_steps), int(check_interval), C.byref(taken),
                                    C.byref(e)), "rq_solve")
        self.fp64 = self.info().precision == L.PREC_FP64  # a mixed new-flavour solve may have promoted
        return taken.value, e.value

    def profile_begin(self):
        self._chk(self.lib.rq_profile_begin(self.ctx), "rq_profile_begin")

    def profile_end(self) -> dict:
        """{kernel class: {launches, ms, bytes, gbs}} since profile_begin (CUDA events)."""
        p = L.Profile()
        self._chk(self.lib.rq_profile_end(self.ctx, C.byref(p)), "rq_profile_end")
        out = {}
        for q, name in enumerate(L.KC_NAMES):
            if p.launches[q]:
                out[name] = {"launches": int(p.launches[q]), "ms": float(p.ms[q]), "bytes": float(p.bytes[q]),
                             "gbs": float(p.bytes[q]) / (float(p.ms[q]) * 1e6) if p.ms[q] > 0 else 0.0}
        return out

    @property
    def kernel_launches(self) -> int:
        return int(self.info().kernel_launches)

    # -- state ----------------------------------------------------------------------------
    def download(self, psi=True, label=True, W=False, P=False):
        S3 = self.S3
        if self.fp64:
            out = {}
            if psi or P:
                u = np.empty(S3, np.float64) if psi else None
                p = np.empty(S3, np.float64) if P else None
                self._chk(self.lib.rq_download_state_f64(self.ctx, _ptr(u), _ptr(p), None), "rq_download_state_f64")
                if psi:
                    out["psi"] = u
                if P:
                    out["P"] = p
            if label or W:
                lab = np.empty(S3, np.int32) if label else None
                w = np.empty(S3, np.float32) if W else None
                self._chk(self.lib.rq_download_state(self.ctx, None, _ptr(lab), _ptr(w), None), "rq_download_state")
                if label:
                    out["label"] = lab
                if W:
                    out["W"] = w
            return out
        u = np.empty(S3, np.float32) if psi else None
        lab = np.empty(S3, np.int32) if label else None
        w = np.empty(S3, np.float32) if W else None
        p = np.empty(S3, np.float32) if P else None
        self._chk(self.lib.rq_download_state(self.ctx, _ptr(u), _ptr(lab), _ptr(w), _ptr(p)), "rq_download_state")
        return {k: v for k, v in (("psi", u), ("label", lab), ("W", w), ("P", p)) if v is not None}

    def download_K(self) -> np.ndarray:
        if self.fp64:
            k = np.empty(self.S3, np.float64)
            self._chk(self.lib.rq_download_state_f64(self.ctx, None, None, _ptr(k)), "rq_download_state_f64")
            return k
        k = np.empty(self.S3, np.float32)
        self._chk(self.lib.rq_download_K(self.ctx, _ptr(k)), "rq_download_K")
        return k

    def upload(self, psi=None, label=None, W=None, P=None):
        cv = lambda a, t: None if a is None else np.ascontiguousarray(np.asarray(a).reshape(-1), dtype=t)
        if self.fp64:
            psi64, P64 = cv(psi, np.float64), cv(P, np.float64)
            if psi64 is not None or P64 is not None:
                self._chk(self.lib.rq_upload_state_f64(self.ctx, _ptr(psi64), _ptr(P64)), "rq_upload_state_f64")
            lab, w = cv(label, np.int32), cv(W, np.float32)
            if lab is not None or w is not None:
                self._chk(self.lib.rq_upload_state(self.ctx, None, _ptr(lab), _ptr(w), None), "rq_upload_state")
            return
        u, lab, w, p = cv(psi, np.float32), cv(label, np.int32), cv(W, np.float32), cv(P, np.float32)
        self._chk(self.lib.rq_upload_state(self.ctx, _ptr(u), _ptr(lab), _ptr(w), _ptr(p)), "rq_upload_state")
