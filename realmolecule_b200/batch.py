"""Batches of independent new-flavour instances with uneven grids (rq_batch_* of include/rq.h).

All instances step in lockstep.  A schedule period of the whole batch is one CUDA-graph replay:
one launch per kernel and phase over the (instance, tile) work lists, or (batch_persistent=1)
ONE persistent cooperative launch whose blocks take chunks of items from a queue, each item
waiting (bounded) only for its own instance's previous phase.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence

import numpy as np

from . import _lib as L
from .context import FLAVORS, PRECISIONS, make_atoms


class Batch:
    def __init__(self, instances: Sequence[dict], precision: str = "mixed", **opts):
        """instances: [{"NN": int, "screen": float, "atoms": [rows]}]; one grid spacing for all."""
        self.lib = L.load()
        n = len(instances)
        cfgs = (L.Config * n)()
        rows: List[dict] = []
        counts = (C.c_int32 * n)()
        for q, inst in enumerate(instances):
            c = cfgs[q]
            c.NN, c.screen = int(inst["NN"]), float(inst["screen"])
            c.flavor, c.precision = FLAVORS["new"], PRECISIONS[precision]
            for k, v in opts.items():
                if v is not None:
                    setattr(c, k, v)
            rows.extend(dict(r, k=r.get("k", inst["NN"] // 2)) for r in inst["atoms"])
            counts[q] = len(inst["atoms"])
        self.counts = list(counts)
        self._atoms = make_atoms(rows)
        h = C.c_void_p()
        L.check(self.lib.rq_batch_create(cfgs, self._atoms, counts, n, C.byref(h)), "rq_batch_create")
        self.b = h
        self.n = n

    def close(self):
        if getattr(self, "b", None):
            self.lib.rq_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st, where):
        if st != L.RQ_OK:
            raise L.RqError(st, where, self.lib.rq_batch_last_error(self.b).decode())

    def set_stream(self, handle):
        self._chk(self.lib.rq_batch_set_stream(self.b, handle), "rq_batch_set_stream")

    def initialize(self):
        self._chk(self.lib.rq_batch_initialize(self.b), "rq_batch_initialize")

    def step(self, n: int = 1):
        self._chk(self.lib.rq_batch_step(self.b, int(n)), "rq_batch_step")

    def synchronize(self):
        self._chk(self.lib.rq_batch_synchronize(self.b), "rq_batch_synchronize")

    def autotune(self) -> dict:
        """rq_batch_autotune: pick the march tile and launch form (timed per step) and the smoother
        sweeps (the cheapest V-cycle converging within 5 % of V(1,1)'s rate); the choice stays in
        the batch.  Returns the choice and every candidate's measurement."""
        r = L.TuneReport()
        self._chk(self.lib.rq_batch_autotune(self.b, C.byref(r)), "rq_batch_autotune")
        tiles = [{"tile": f"{1 << (r.tile[i] & 0xff)}x{256 >> (r.tile[i] & 0xff)}x{r.tile[i] >> 8}",
                  "batch_tile": r.tile[i], "persistent": r.persistent[i], "ms_per_step": r.ms_per_step[i]}
                 for i in range(r.n_tile)]
        smooth = [{"mg_pre": r.pre[i], "mg_post": r.post[i], "mg_coarse_sweeps": r.coarse_sweeps[i], "rho": r.rho[i],
                   "ms_per_cycle": r.ms_per_cycle[i]} for i in range(r.n_smooth)]
        best = {}
        if r.n_tile:
            t = tiles[r.best_tile]
            best.update(batch_tile=t["batch_tile"], batch_persistent=t["persistent"])
        if r.n_smooth:
            m = smooth[r.best_smooth]
            best.update(mg_pre=m["mg_pre"], mg_post=m["mg_post"], mg_coarse_sweeps=m["mg_coarse_sweeps"])
        return {"config": best, "tiles": tiles, "smoothers": smooth}

    def set_wait(self, limit_ns: int, extra_arrivals: int = 0):
        """Bound of the persistent launch's waits; extra_arrivals > 0 makes every wait run out (the
        next readout raises RqError with RQ_ETIMEOUT)."""
        self._chk(self.lib.rq_batch_set_wait(self.b, int(limit_ns), int(extra_arrivals)), "rq_batch_set_wait")

    def energy(self) -> np.ndarray:
        out = np.zeros((self.n, L.ENERGY_LEN))
        self._chk(self.lib.rq_batch_energy(self.b, out.ctypes.data), "rq_batch_energy")
        return out

    def forces(self) -> List[np.ndarray]:
        F = np.zeros((sum(self.counts), 3))
        self._chk(self.lib.rq_batch_forces(self.b, F.ctypes.data), "rq_batch_forces")
        return np.split(F, np.cumsum(self.counts)[:-1])

    def solve(self, tol_dE: float, max_steps: int, check_interval: int = 100):
        conv = np.zeros(self.n, np.int32)
        E = np.zeros(self.n)
        self._chk(self.lib.rq_batch_solve(self.b, float(tol_dE), int(max_steps), int(check_interval),
                                          conv.ctypes.data, E.ctypes.data), "rq_batch_solve")
        return conv, E

    def info(self):
        n, tp, ip, kl = C.c_int32(), C.c_int64(), C.c_int64(), C.c_int64()
        self._chk(self.lib.rq_batch_info(self.b, C.byref(n), C.byref(tp), C.byref(ip), C.byref(kl)), "rq_batch_info")
        return {"instances": n.value, "points": tp.value, "interior_points": ip.value, "kernel_launches": kl.value}


def _main(argv=None):
    """Step the seeded 96-water-cluster batch (realmolecule_b200.configs.clusters96) on cuda:0.

    python -m realmolecule_b200.batch [--instances N] [--steps K] [--precision mixed|fp64] [--persistent]
    Prints the batch size and the wall time of the K steps (after initialisation and 40 warm-up
    steps, which capture the periods)."""
    import argparse
    import time

    from . import configs
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--instances", type=int, default=96)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--precision", default="mixed", choices=sorted(PRECISIONS))
    ap.add_argument("--persistent", action="store_true", help="one persistent launch per period")
    a = ap.parse_args(argv)
    geoms = configs.clusters96()[:a.instances]
    b = Batch([{"NN": g.NN, "screen": g.screen, "atoms": configs.to_domain_atoms(g)} for g in geoms],
              precision=a.precision, label_until=1, batch_persistent=1 if a.persistent else 0)
    b.initialize()
    b.step(40)
    b.synchronize()
    t0 = time.perf_counter()
    b.step(a.steps)
    b.synchronize()
    dt = time.perf_counter() - t0
    print({**b.info(), "steps": a.steps, "ms_per_step": dt / max(1, a.steps) * 1e3}, flush=True)
    b.close()


if __name__ == "__main__":
    _main()
