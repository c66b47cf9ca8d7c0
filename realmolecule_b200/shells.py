"""The atom.js per-shell solver on the GPU (rq_shells_* of include/rq.h).

Drop-in for atom.js's module (atom.js:1-346): the constructor takes the page's globals
(USER_NN, USER_SCREEN, USER_Z_KERNEL, USER_SHELLS, USER_D, USER_POISSON) and ``physicsStep()``
returns the same dict.  Shells use atom.js's idiom: ``{"ne": 1, "Rmax": 1.0, "Zeff": 2}`` plus
optional ``split="halfspace"``, ``halfIndex``, ``outerHalf``, ``fixedW``.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Sequence

import numpy as np

from . import _lib as L


def _shells(shells: Sequence[dict]):
    arr = (L.Shell * len(shells))()
    for q, sh in enumerate(shells):
        arr[q].ne = sh.get("ne", 1)
        arr[q].Rmax = sh.get("Rmax", 0.0) or 0.0
        arr[q].Zeff = sh["Zeff"]
        arr[q].split = 1 if sh.get("split") == "halfspace" else 0
        arr[q].half_index = int(sh.get("halfIndex", 0))
        arr[q].outer_half = int(bool(sh.get("outerHalf", False)))
        arr[q].fixed_w = int(bool(sh.get("fixedW", False)))
    return arr


class AtomShells:
    def __init__(self, NN: int = 100, screen: float = 10.0, Z_kernel: float = 2.0,
                 shells: Sequence[dict] = ({"ne": 1, "Rmax": 1.0, "Zeff": 2}, {"ne": 1, "Rmax": 5.0, "Zeff": 1}),
                 d: float = 0.1, poisson: str = "multigrid"):
        self.lib = L.load()
        cfg = L.ShellsConfig()
        cfg.NN, cfg.screen, cfg.Z_kernel, cfg.d = int(NN), float(screen), float(Z_kernel), float(d)
        cfg.poisson = 1 if poisson == "simultaneous" else 0
        self._sh = _shells(shells)
        self.n_shells = len(shells)
        self.NN, self.S = int(NN), int(NN) + 1
        self.S3 = self.S ** 3
        h = C.c_void_p()
        L.check(self.lib.rq_shells_create(C.byref(cfg), self._sh, self.n_shells, C.byref(h)), "rq_shells_create")
        self.s = h

    def close(self):
        if getattr(self, "s", None):
            self.lib.rq_shells_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st, where):
        if st != L.RQ_OK:
            raise L.RqError(st, where, self.lib.rq_shells_last_error(self.s).decode())

    def step(self, n: int = 1) -> Dict:
        """n physicsStep() calls; the dict of the last one (atom.js:341-342)."""
        E = np.zeros(4)
        ps = np.zeros((self.n_shells, 5))
        self._chk(self.lib.rq_shells_step(self.s, int(n), E.ctypes.data, ps.ctypes.data), "rq_shells_step")
        return {"E": E[0], "E_T": E[1], "E_eK": E[2], "E_ee": E[3], "ET_m": ps[:, 0].tolist(),
                "Eee_m": ps[:, 1].tolist(), "EeK_m": ps[:, 2].tolist(), "nrm_m": ps[:, 3].tolist(),
                "eig": ps[:, 4].tolist()}

    def physicsStep(self) -> Dict:  # noqa: N802 -- atom.js's name
        return self.step(1)

    def fields(self, shell: int) -> Dict[str, np.ndarray]:
        U, W, P = (np.empty(self.S3, np.float32) for _ in range(3))
        self._chk(self.lib.rq_shells_download(self.s, int(shell), U.ctypes.data, W.ctypes.data, P.ctypes.data),
                  "rq_shells_download")
        return {"U": U, "W": W, "P": P}

    def set_fields(self, shell: int, U=None, W=None, P=None):
        cv = lambda a: None if a is None else np.ascontiguousarray(a, np.float32).reshape(-1)
        U, W, P = cv(U), cv(W), cv(P)
        ptr = lambda a: None if a is None else a.ctypes.data
        self._chk(self.lib.rq_shells_upload(self.s, int(shell), ptr(U), ptr(W), ptr(P)), "rq_shells_upload")

    @property
    def kernel_launches(self) -> int:
        n = C.c_int64()
        self._chk(self.lib.rq_shells_info(self.s, C.byref(n)), "rq_shells_info")
        return n.value
