"""The mol_fast.js multi-field solver on the GPU (rq_mf_* of include/rq.h).

Drop-in for mol_fast.js's module (mol_fast.js:12-1651): the constructor takes the page's
globals (``USER_NUCLEI``, ``USER_NN``, ``USER_SCREEN``, ``USER_NORM_TARGETS``, ... as keyword
arguments, or a dict of them through :meth:`MolFast.from_page`), and the host logic around the
GPU work is the page's own: ``doSteps(n)`` (energies and dipole from the frame's last
reduction), ``computeForces()`` (the device's Hartree gradient plus the softened nuclear
repulsion), ``stepNuclei()`` (damped velocity update, moves below 1e-4 cells ignored, K rebuilt
after a move) and ``frame()`` = one ``draw()`` tick.  The slice the page draws is returned by
``extract()`` as a plain array.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib as L

SPLIT_CODES = {"sphere": 0, "hemi": 2, "third": 3, "tetra": 4, "hemi_third": 5}
PROTON_MASS = 1836


def normalize_nuclei(raw: Sequence[dict]) -> List[dict]:
    """The page's nucleus records (mol_fast.js:28-40) with their defaults."""
    out = []
    for n in raw:
        Z = n["Z"]
        out.append({
            "i": n["i"], "j": n["j"], "k": n["k"], "Z": Z,
            "rc": n.get("rc") or 0, "r_out": n.get("r_out") or 0, "tilt_y": n.get("tilt_y") or 0,
            "tilt_x": n.get("tilt_x") or 0, "hs": n.get("hs") or 0, "fixed": n.get("fixed") is True,
            "z_init": n["z_init"] if n.get("z_init") is not None else (Z if Z > 0 else 1),
            "split": n.get("split") or "sphere", "split_idx": n.get("split_idx") or 0,
            "split_axis": list(n.get("split_axis") or [1, 0, 0]),
            "split_fix": n["split_fix"] if n.get("split_fix") is not None else True,
        })
    return out


class MolFast:
    """One mol_fast.js page on the GPU.  Nuclear positions are grid coordinates (i, j, k)."""

    def __init__(self, nuclei: Sequence[dict], NN: int = 200, screen: float = 15.0,
                 norm_targets: Optional[Sequence[float]] = None, steps_per_frame: int = 500,
                 max_steps: int = 100000, shell_mode: bool = False, vcycle: bool = True, vcycle_interval: int = 50,
                 coarse_iters: int = 10, kinetic_coeff: float = 0.5, kc_multi: float = 1.0,
                 beta_pauli: float = 0.0, field_x: float = 0.0, alpha_tf: float = 0.0, full_self: bool = False,
                 r_out_release_step: Optional[int] = None, line_j_offset: float = 0.0, dt_nuc: float = 2.0,
                 nuc_damping: float = 0.9, force_scale: float = 1.0, mass: Optional[Sequence[float]] = None,
                 dynamics: bool = False):
        if len(nuclei) > 16:
            raise ValueError(f"mol_fast: MAX_ATOMS = 16, got {len(nuclei)}")
        if NN % 2:
            raise ValueError("mol_fast: NN must be even for V-cycle")
        self.nuclei = normalize_nuclei(nuclei)
        self.n = len(self.nuclei)
        self.NN, self.S = int(NN), int(NN) + 1
        self.S3 = self.S ** 3
        self.N2 = round(NN / 2)
        self.screen = float(screen)
        self.hv = self.screen / NN
        self.h2v = self.hv * self.hv
        self.norm_targets = list(norm_targets) if norm_targets is not None else [1] * self.n
        self.steps_per_frame = int(steps_per_frame)
        self.max_steps = int(max_steps)
        self.dt_nuc, self.nuc_damping, self.force_scale = float(dt_nuc), float(nuc_damping), float(force_scale)
        self.nuc_mass = list(mass) if mass is not None else [max(1, a["Z"]) * PROTON_MASS for a in self.nuclei]
        self.dynamics = bool(dynamics)
        self.nuc_vel = [[0.0, 0.0, 0.0] for _ in range(self.n)]
        self.nuc_force = [[0.0, 0.0, 0.0] for _ in range(self.n)]
        self.tStep = 0
        self.E = self.E_T = self.E_eK = self.E_ee = 0.0
        self.dipole = [0.0, 0.0, 0.0]
        self.dipoleMag = 0.0
        self.sums = np.zeros(self.n + 6, np.float32)

        cfg = L.MfConfig()
        cfg.NN, cfg.shell_mode, cfg.vcycle = self.NN, int(bool(shell_mode)), int(bool(vcycle))
        cfg.vcycle_interval, cfg.coarse_iters = int(vcycle_interval), int(coarse_iters)
        cfg.r_out_release_step = -1 if r_out_release_step is None else int(r_out_release_step)
        cfg.full_self = int(bool(full_self))
        cfg.screen, cfg.kinetic_coeff, cfg.kc_multi = self.screen, float(kinetic_coeff), float(kc_multi)
        cfg.beta_pauli, cfg.field_x, cfg.alpha_tf = float(beta_pauli), float(field_x), float(alpha_tf)
        cfg.line_j_offset = float(line_j_offset)
        arr = (L.MfNucleus * self.n)()
        for q, a in enumerate(self.nuclei):
            r = arr[q]
            r.i, r.j, r.k, r.Z = a["i"], a["j"], a["k"], a["Z"]
            r.rc, r.r_out, r.tilt_y, r.tilt_x, r.hs = a["rc"], a["r_out"], a["tilt_y"], a["tilt_x"], a["hs"]
            r.z_init, r.norm_target = a["z_init"], self.norm_targets[q]
            r.split_axis[:] = [float(v) for v in a["split_axis"]]
            r.split = SPLIT_CODES.get(a["split"], 0)
            r.split_idx, r.split_fix = int(a["split_idx"]), int(bool(a["split_fix"]))
        self.lib = L.load()
        h = C.c_void_p()
        L.check(self.lib.rq_mf_create(C.byref(cfg), arr, self.n, C.byref(h)), "rq_mf_create")
        self.s = h
        self.computeEKK()

    @classmethod
    def from_page(cls, g: Dict) -> "MolFast":
        """Build from a dict of the page's window.USER_* globals (mol_fast.js:14-104)."""
        keys = {"USER_NN": "NN", "USER_SCREEN": "screen", "USER_NORM_TARGETS": "norm_targets",
                "USER_STEPS_PER_FRAME": "steps_per_frame", "USER_STEPS": "max_steps",
                "USER_SHELL_MODE": "shell_mode", "USER_VCYCLE_INTERVAL": "vcycle_interval",
                "USER_COARSE_ITERS": "coarse_iters", "USER_KINETIC_COEFF": "kinetic_coeff",
                "USER_KC_MULTI": "kc_multi", "USER_BETA_PAULI": "beta_pauli", "USER_FIELD_X": "field_x",
                "USER_ALPHA_TF": "alpha_tf", "USER_FULL_SELF": "full_self",
                "USER_R_OUT_RELEASE_STEP": "r_out_release_step", "USER_LINE_J_OFFSET": "line_j_offset",
                "USER_DT_NUC": "dt_nuc", "USER_NUC_DAMPING": "nuc_damping", "USER_FORCE_SCALE": "force_scale",
                "USER_MASS": "mass", "USER_DYNAMICS": "dynamics"}
        kw = {v: g[k] for k, v in keys.items() if g.get(k) is not None}
        if "USER_VCYCLE" in g:
            kw["vcycle"] = g["USER_VCYCLE"] is not False
        if kw.get("shell_mode") is not None:
            kw["shell_mode"] = kw["shell_mode"] is True
        return cls(g["USER_NUCLEI"], **kw)

    # ---- lifetime ---------------------------------------------------------------------------
    def close(self):
        if getattr(self, "s", None):
            self.lib.rq_mf_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st, where):
        if st != L.RQ_OK:
            raise L.RqError(st, where, self.lib.rq_mf_last_error(self.s).decode())

    # ---- the page's host logic ------------------------------------------------------------------
    def computeEKK(self) -> float:  # noqa: N802 -- mol_fast.js:1326-1337
        E = 0.0
        nu, hv = self.nuclei, self.hv
        for a in range(self.n):
            for b in range(a + 1, self.n):
                dx = (nu[a]["i"] - nu[b]["i"]) * hv
                dy = (nu[a]["j"] - nu[b]["j"]) * hv
                dz = (nu[a]["k"] - nu[b]["k"]) * hv
                r = math.sqrt(dx * dx + dy * dy + dz * dz)
                if r > 0:
                    E += nu[a]["Z"] * nu[b]["Z"] / r
        self.E_KK = E
        return E

    def doSteps(self, n: int) -> Dict:  # noqa: N802 -- mol_fast.js:1237-1322
        self._chk(self.lib.rq_mf_step(self.s, int(n), self.sums.ctypes.data), "rq_mf_step")
        s, ne = self.sums, self.n
        self.E_T, self.E_eK, self.E_ee = float(s[ne]), float(s[ne + 1]), float(s[ne + 2])
        self.E = self.E_T + self.E_eK + self.E_ee + self.E_KK
        dn = [0.0, 0.0, 0.0]
        for a in self.nuclei:
            dn[0] += a["Z"] * (a["i"] - self.N2) * self.hv
            dn[1] += a["Z"] * (a["j"] - self.N2) * self.hv
            dn[2] += a["Z"] * (a["k"] - self.N2) * self.hv
        self.dipole = [dn[0] + float(s[ne + 3]), dn[1] + float(s[ne + 4]), dn[2] + float(s[ne + 5])]
        self.dipoleMag = math.hypot(*self.dipole)
        self.tStep += n
        if not math.isfinite(self.E):
            raise FloatingPointError(f"numerical instability at step {self.tStep}")
        return self.energies()

    def energies(self) -> Dict:
        return {"E": self.E, "E_T": self.E_T, "E_eK": self.E_eK, "E_ee": self.E_ee, "E_KK": self.E_KK,
                "dipole": list(self.dipole), "dipoleMag": self.dipoleMag,
                "norms": [float(v) for v in self.sums[:self.n]]}

    def computeForces(self) -> List[List[float]]:  # noqa: N802 -- mol_fast.js:1339-1373
        fd = np.zeros(3 * self.n, np.float32)
        self._chk(self.lib.rq_mf_forces(self.s, fd.ctypes.data), "rq_mf_forces")
        nu, hv, h2v = self.nuclei, self.hv, self.h2v
        for a in range(self.n):
            f = [float(fd[3 * a]), float(fd[3 * a + 1]), float(fd[3 * a + 2])]
            for b in range(self.n):
                if b == a:
                    continue
                dx = (nu[a]["i"] - nu[b]["i"]) * hv
                dy = (nu[a]["j"] - nu[b]["j"]) * hv
                dz = (nu[a]["k"] - nu[b]["k"]) * hv
                r2 = dx * dx + dy * dy + dz * dz + h2v
                inv_r3 = 1 / (r2 * math.sqrt(r2))
                pref = nu[a]["Z"] * nu[b]["Z"] * inv_r3
                f[0] += pref * dx
                f[1] += pref * dy
                f[2] += pref * dz
            self.nuc_force[a] = f
        return self.nuc_force

    def stepNuclei(self) -> bool:  # noqa: N802 -- mol_fast.js:1375-1410
        dt, moved = self.dt_nuc, False
        for a, nuc in enumerate(self.nuclei):
            if nuc["Z"] <= 0 or nuc["fixed"]:
                continue
            m = self.nuc_mass[a]
            v = self.nuc_vel[a]
            for d in range(3):
                v[d] = self.nuc_damping * (v[d] + dt * self.force_scale * self.nuc_force[a][d] / m)
            di, dj, dk = (v[0] * dt) / self.hv, (v[1] * dt) / self.hv, (v[2] * dt) / self.hv
            if abs(di) > 0.0001 or abs(dj) > 0.0001 or abs(dk) > 0.0001:
                nuc["i"] += di
                nuc["j"] += dj
                nuc["k"] += dk
                moved = True
        if moved:
            self.set_positions([(a["i"], a["j"], a["k"]) for a in self.nuclei])
        return moved

    def set_positions(self, ijk):
        """Moved nuclei: parameters rewritten, E_KK recomputed and K rebuilt on the device."""
        arr = np.ascontiguousarray(np.asarray(ijk, np.float64).reshape(self.n, 3))
        for a, nuc in enumerate(self.nuclei):
            nuc["i"], nuc["j"], nuc["k"] = float(arr[a, 0]), float(arr[a, 1]), float(arr[a, 2])
        self.computeEKK()
        self._chk(self.lib.rq_mf_set_positions(self.s, arr.ctypes.data), "rq_mf_set_positions")

    def frame(self) -> Dict:
        """One draw() tick (mol_fast.js:1434-1446): doSteps, computeForces, then stepNuclei
        while dynamics is on."""
        if self.tStep >= self.max_steps:
            return self.energies()
        out = self.doSteps(self.steps_per_frame)
        self.computeForces()
        if self.dynamics:
            self.stepNuclei()
        return out

    # ---- buffers ------------------------------------------------------------------------------
    def extract(self) -> np.ndarray:
        """The page's slice buffer (mol_fast.js:595-640): 3 n S^2 floats."""
        out = np.zeros(3 * self.n * self.S * self.S, np.float32)
        self._chk(self.lib.rq_mf_extract(self.s, out.ctypes.data), "rq_mf_extract")
        return out

    def fields(self, m: int) -> Dict[str, np.ndarray]:
        U, W, P = (np.empty(self.S3, np.float32) for _ in range(3))
        self._chk(self.lib.rq_mf_download(self.s, int(m), U.ctypes.data, W.ctypes.data, P.ctypes.data),
                  "rq_mf_download")
        return {"U": U, "W": W, "P": P}

    def set_fields(self, m: int, U=None, W=None, P=None):
        cv = lambda a: None if a is None else np.ascontiguousarray(a, np.float32).reshape(-1)
        U, W, P = cv(U), cv(W), cv(P)
        ptr = lambda a: None if a is None else a.ctypes.data
        self._chk(self.lib.rq_mf_upload(self.s, int(m), ptr(U), ptr(W), ptr(P)), "rq_mf_upload")

    def K(self) -> np.ndarray:
        K = np.empty(self.S3, np.float32)
        self._chk(self.lib.rq_mf_download_K(self.s, K.ctypes.data), "rq_mf_download_K")
        return K

    @property
    def kernel_launches(self) -> int:
        n, t = C.c_int64(), C.c_int64()
        self._chk(self.lib.rq_mf_info(self.s, C.byref(n), C.byref(t)), "rq_mf_info")
        return n.value


def _main(argv=None):
    """Run a mol_fast.js page (realmolecule_b200.configs) on cuda:0.

    python -m realmolecule_b200.mol_fast [--page ch4|h2] [--steps K] [--frames F]
    Prints the energies after F frames of K steps (each followed by computeForces)."""
    import argparse
    import time

    from . import configs
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--page", default="ch4", choices=["ch4", "h2"])
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--frames", type=int, default=1)
    a = ap.parse_args(argv)
    cfg = configs.mol_fast_ch4_page() if a.page == "ch4" else configs.mol_fast_h2_page()
    mf = MolFast(**cfg)
    t0 = time.perf_counter()
    for _ in range(a.frames):
        mf.doSteps(a.steps)
        mf.computeForces()
    dt = time.perf_counter() - t0
    print({**mf.energies(), "steps": a.steps * a.frames, "ms_per_step": dt / max(1, a.steps * a.frames) * 1e3},
          flush=True)
    mf.close()


if __name__ == "__main__":
    _main()
