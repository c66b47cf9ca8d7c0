"""The realqm_rb.js red-black multi-field solver on the GPU (rq_rb_* of include/rq.h).

Drop-in for realqm_rb.js (realqm_rb.js:1-1222): the constructor takes the page's globals
(``USER_NUCLEI``, ``USER_NN``, ``USER_SCREEN``, ``USER_NELEC``, ``USER_NORM_TARGETS``, ...)
as keyword arguments or a dict through :meth:`RealqmRb.from_page`; ``doSteps(n)``,
``computeEnergy()`` and ``extractSlice()`` keep the page's names, and ``frame()`` is one
``draw()`` tick (STEPS_PER_FRAME steps, energies every third frame).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib as L


def default_nuclei(NN: int, d_cells: int = 0) -> List[dict]:
    """The page's two-nucleus default (realqm_rb.js:40-49)."""
    N2 = NN // 2
    half = math.floor(d_cells / 2 + 0.5)
    return [{"i": N2 - half, "j": N2, "k": N2, "Z": 1, "rc": 0, "ne": 1},
            {"i": N2 + half, "j": N2, "k": N2, "Z": 1, "rc": 0, "ne": 1}]


class RealqmRb:
    """One realqm_rb.js page on the GPU.  Nuclear positions are grid coordinates (i, j, k)."""

    def __init__(self, nuclei: Optional[Sequence[dict]] = None, NN: int = 100, screen: float = 8.0,
                 nelec: Optional[int] = None, norm_targets: Optional[Sequence[float]] = None,
                 max_steps: int = 10000, d_cells: int = 0, no_nuc_repulsion: bool = False):
        raw = list(nuclei) if nuclei is not None else default_nuclei(NN, d_cells)
        self.nuclei = [dict(n, ne=1 if n.get("ne") is None else n["ne"], rc=n.get("rc") or 0) for n in raw]
        ne_sum = sum(int(n["ne"]) for n in self.nuclei)
        self.nelec = ne_sum if nelec is None else int(nelec)
        if self.nelec != ne_sum:
            raise ValueError(f"realqm_rb: USER_NELEC = {self.nelec} but the nuclei carry {ne_sum} electrons")
        self.NN, self.S = int(NN), int(NN) + 1
        self.S3 = self.S ** 3
        self.screen = float(screen)
        self.h = self.screen / NN
        self.h2 = self.h * self.h
        self.max_steps = int(max_steps)
        self.steps_per_frame = 10 if NN <= 100 else (6 if NN <= 150 else (4 if NN <= 200 else 2))
        self.stepCount = 0
        self.frame_count = 0
        self.E_T = self.E_eK = self.E_ee = self.E_tot = 0.0
        self.V_KK = 0.0
        if not no_nuc_repulsion:  # realqm_rb.js:57-68
            nu = self.nuclei
            for a in range(len(nu)):
                for b in range(a + 1, len(nu)):
                    dx = (nu[a]["i"] - nu[b]["i"]) * self.h
                    dy = (nu[a]["j"] - nu[b]["j"]) * self.h
                    dz = (nu[a]["k"] - nu[b]["k"]) * self.h
                    r = math.sqrt(dx * dx + dy * dy + dz * dz)
                    if r > 0:
                        self.V_KK += nu[a]["Z"] * nu[b]["Z"] / math.sqrt(r * r + self.h2)
        cfg = L.RbConfig()
        cfg.NN, cfg.screen = self.NN, self.screen
        arr = (L.RbNucleus * len(self.nuclei))()
        for q, a in enumerate(self.nuclei):
            arr[q].i, arr[q].j, arr[q].k, arr[q].Z = a["i"], a["j"], a["k"], a["Z"]
            arr[q].rc, arr[q].rc_excl, arr[q].ne = a["rc"], a.get("rc_excl") or 0.0, int(a["ne"])
        tg = None
        if norm_targets is not None:  # indexed by electron, like the page (a missing entry is NaN)
            tg = np.array([float(norm_targets[m]) if m < len(norm_targets) and norm_targets[m] is not None
                           else float("nan") for m in range(self.nelec)])
        self.norm_targets = tg
        self.lib = L.load()
        h = C.c_void_p()
        L.check(self.lib.rq_rb_create(C.byref(cfg), arr, len(self.nuclei), None if tg is None else tg.ctypes.data,
                                      C.byref(h)), "rq_rb_create")
        self.s = h

    @classmethod
    def from_page(cls, g: Dict) -> "RealqmRb":
        """Build from a dict of the page's window.* globals (realqm_rb.js:8-55)."""
        return cls(g.get("USER_NUCLEI"), NN=g.get("USER_NN") or 100, screen=g.get("USER_SCREEN") or 8,
                   nelec=g.get("USER_NELEC") or 2, norm_targets=g.get("USER_NORM_TARGETS"),
                   max_steps=g.get("USER_STEPS") or 10000, d_cells=g.get("USER_D") or 0,
                   no_nuc_repulsion=bool(g.get("NO_NUC_REPULSION")))

    def close(self):
        if getattr(self, "s", None):
            self.lib.rq_rb_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st, where):
        if st != L.RQ_OK:
            raise L.RqError(st, where, self.lib.rq_rb_last_error(self.s).decode())

    def doSteps(self, n: int):  # noqa: N802 -- realqm_rb.js:891-965
        self._chk(self.lib.rq_rb_step(self.s, int(n)), "rq_rb_step")
        self.stepCount += n

    def computeEnergy(self) -> Dict:  # noqa: N802 -- realqm_rb.js:982-1045
        e = np.zeros(3)
        self._chk(self.lib.rq_rb_energy(self.s, e.ctypes.data), "rq_rb_energy")
        self.E_T, self.E_eK, self.E_ee = float(e[0]), float(e[1]), float(e[2])
        self.E_tot = self.E_T + self.E_eK + self.E_ee + self.V_KK
        return {"E_T": self.E_T, "E_eK": self.E_eK, "E_ee": self.E_ee, "V_KK": self.V_KK, "E_tot": self.E_tot}

    def extractSlice(self) -> np.ndarray:  # noqa: N802 -- realqm_rb.js:1047-1066
        out = np.empty(self.S * self.S * (3 * self.nelec + 1), np.float32)
        self._chk(self.lib.rq_rb_slice(self.s, out.ctypes.data), "rq_rb_slice")
        return out

    def frame(self) -> Dict:
        """One draw() tick (realqm_rb.js:1093-1146): STEPS_PER_FRAME steps while stepCount < MAX_STEPS,
        then on every third frame (and when done) the energies."""
        self.frame_count += 1
        if self.stepCount < self.max_steps:
            self.doSteps(self.steps_per_frame)
        if self.frame_count % 3 == 0 or self.stepCount >= self.max_steps:
            self.computeEnergy()
        return {"stepCount": self.stepCount, "maxSteps": self.max_steps, "E_T": self.E_T, "E_eK": self.E_eK,
                "E_ee": self.E_ee, "V_KK": self.V_KK, "E_tot": self.E_tot, "done": self.stepCount >= self.max_steps}

    def fields(self, m: int) -> Dict[str, np.ndarray]:
        U, W, P = (np.empty(self.S3, np.float32) for _ in range(3))
        self._chk(self.lib.rq_rb_download(self.s, int(m), U.ctypes.data, W.ctypes.data, P.ctypes.data),
                  "rq_rb_download")
        return {"U": U, "W": W, "P": P}

    def set_fields(self, m: int, U=None, W=None, P=None):
        cv = lambda a: None if a is None else np.ascontiguousarray(a, np.float32).reshape(-1)
        U, W, P = cv(U), cv(W), cv(P)
        ptr = lambda a: None if a is None else a.ctypes.data
        self._chk(self.lib.rq_rb_upload(self.s, int(m), ptr(U), ptr(W), ptr(P)), "rq_rb_upload")

    def K(self) -> np.ndarray:
        K = np.empty(self.S3, np.float32)
        self._chk(self.lib.rq_rb_download_K(self.s, K.ctypes.data), "rq_rb_download_K")
        return K

    @property
    def kernel_launches(self) -> int:
        n, t = C.c_int64(), C.c_int64()
        self._chk(self.lib.rq_rb_info(self.s, C.byref(n), C.byref(t)), "rq_rb_info")
        return n.value


def _main(argv=None):
    """Run realqm_rb.js's direct H2 page (realmolecule_b200.configs.realqm_rb_h2_page) on cuda:0.

    python -m realmolecule_b200.realqm_rb [--steps K]
    Prints the energies after K steps."""
    import argparse
    import time

    from . import configs
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--steps", type=int, default=100)
    a = ap.parse_args(argv)
    g = RealqmRb(**configs.realqm_rb_h2_page())
    t0 = time.perf_counter()
    g.doSteps(a.steps)
    dt = time.perf_counter() - t0
    print({**g.computeEnergy(), "steps": a.steps, "ms_per_step": dt / max(1, a.steps) * 1e3}, flush=True)
    g.close()


if __name__ == "__main__":
    _main()
