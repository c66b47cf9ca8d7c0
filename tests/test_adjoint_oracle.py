"""The FP64 restatement of the new flavour's adjoint (oracle/nm_adjoint.py) against central finite
differences of the oracle's own forward schedule (oracle.NewMethodDriver), on the CPU.

E(R) is the energy read out after N warm-started steps from one fixed, non-converged state with
the labels frozen; every finite difference restarts from that state in the same schedule phase.
Bars: 1e-7 Ha/bohr for the nuclear forces (delta = 1e-4 bohr), 1e-7 relative for the
directional derivative along an external potential.  The Hellmann-Feynman force alone differs
from the finite differences by ~1e-3 here (the state is not converged), so the reverse sweep is
what the agreement measures.
"""
import numpy as np

import oracle as orc
import nm_adjoint as adj

N_STEPS = 16
DELTA = 1e-4


def _h2(NN=16, h=0.45, R=1.4):
    N2 = NN / 2
    d = R / 2 / h
    return NN, NN * h, [
        {"i": N2 - d, "j": N2, "k": N2 + 0.2, "Z": 0.0, "Z_nuc": 1.0},
        {"i": N2 + d, "j": N2 + 0.3, "k": N2, "Z": 0.0, "Z_nuc": 1.0},
        {"i": N2 - d + 0.05, "j": N2, "k": N2, "Z": 1.0, "Z_nuc": 0.0},
        {"i": N2 + d - 0.05, "j": N2, "k": N2, "Z": 1.0, "Z_nuc": 0.0}]


def _start():
    NN, scr, rows = _h2()
    drv = orc.NewMethodDriver(NN, scr, rows, label_until=40)
    drv.initialize()
    for _ in range(60):
        drv.step()
    drv.ready()
    return drv, rows, (drv.U.copy(), drv.P.copy(), drv.steps_done)


def _restore(drv, st, rows):
    drv.U[:], drv.P[:] = st[0], st[1]
    drv.steps_done, drv.age = st[2], 0
    drv.set_positions(rows)


def _energy(drv, st, rows, v=None):
    _restore(drv, st, rows)
    if v is not None:
        drv.K += v
    for _ in range(N_STEPS):
        drv.step()
    return drv.energy()["E"]


def _nuclear_forces(rows, h):
    xyz = np.array([[r["i"] * h, r["j"] * h, r["k"] * h] for r in rows])
    Z = np.array([r["Z_nuc"] for r in rows])
    F = np.zeros_like(xyz)
    for a in range(len(rows)):
        for b in range(len(rows)):
            if a != b and Z[a] > 0 and Z[b] > 0:
                d = xyz[a] - xyz[b]
                F[a] += Z[a] * Z[b] * d / np.linalg.norm(d) ** 3
    return F


def test_oracle_adjoint_forces_match_finite_differences():
    drv, rows, st = _start()
    _restore(drv, st, rows)
    Fhf = drv.forces()  # the Hellmann-Feynman force at the starting state, for contrast below
    _restore(drv, st, rows)
    E0, Fe, _ = adj.gradient(drv, N_STEPS)
    Fn = _nuclear_forces(rows, drv.h)
    F = Fe + Fn
    assert abs(E0 - _energy(drv, st, rows)) < 1e-12 * abs(E0)  # recording leaves the forward as it is
    gap = 0.0
    for a in (0, 1):
        for ax in range(3):
            E = []
            for sgn in (1, -1):
                r2 = [dict(r) for r in rows]
                r2[a]["ijk"[ax]] += sgn * DELTA / drv.h
                E.append(_energy(drv, st, r2))
            fd = -(E[0] - E[1]) / (2 * DELTA)
            assert abs(fd - F[a, ax]) < 1e-7, (a, ax, fd, F[a, ax])
            gap = max(gap, abs(fd - Fhf[a, ax] - Fn[a, ax]))
    assert gap > 1e-4  # a non-converged state: the reverse sweep carries a real correction


def test_oracle_adjoint_potential_gradient_matches_finite_differences():
    drv, rows, st = _start()
    S = drv.S
    x = (np.arange(S) - S / 2) * drv.h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    w = (np.exp(-((X - 0.5) ** 2 + Y ** 2 + (Z + 0.4) ** 2) / 2.0) * (1 + 0.3 * X)).reshape(-1)
    _restore(drv, st, rows)
    _, _, gK = adj.gradient(drv, N_STEPS)
    eps = 1e-5
    fd = (_energy(drv, st, rows, eps * w) - _energy(drv, st, rows, -eps * w)) / (2 * eps)
    ad = float(np.dot(gK, w))
    assert abs(fd - ad) < 1e-7 * max(1.0, abs(fd)), (fd, ad)
