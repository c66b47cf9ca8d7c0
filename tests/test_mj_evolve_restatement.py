"""A second, pure-Python restatement of molecule.js's evolveBoundary (molecule.js:426-540) with
locked groups (:490-503) and shell-split sectors (:197-226, :514-533), written from the shader
text independently of oracle/rq_oracle.c and compared with it bit for bit on small random grids
(CPU).  The GPU kernel is compared with the C restatement in test_gpu_mj.py."""
import math

import numpy as np
import pytest

import oracle as orc

f32 = np.float32


def in_split(d, r, sp):
    """inSplitAtom in f32 steps; atan2 in double rounded once to f32 (as both restatements)."""
    st = sp["type"]
    if st <= 1 or r < f32(1e-6):
        return True
    ax = [f32(x) for x in sp["axis"]]
    axL = max(f32(math.sqrt(f32(f32(ax[0] * ax[0]) + f32(ax[1] * ax[1])) + f32(ax[2] * ax[2]))), f32(1e-12))
    a = [f32(x / axL) for x in ax]
    dotp = f32(f32(f32(d[0] * a[0]) + f32(d[1] * a[1])) + f32(d[2] * a[2]))
    if st == 2:
        return dotp < 0 if sp["idx"] == 0 else dotp >= 0
    if st == 3:
        p = [f32(d[c] - f32(dotp * a[c])) for c in range(3)]
        e1 = [a[1], f32(-a[0]), f32(0)] if abs(a[2]) < f32(0.9) else [f32(0), a[2], f32(-a[1])]
        e1L = max(f32(math.sqrt(f32(f32(f32(e1[0] * e1[0]) + f32(e1[1] * e1[1])) + f32(e1[2] * e1[2])))), f32(1e-12))
        e1 = [f32(x / e1L) for x in e1]
        e2 = [f32(f32(a[1] * e1[2]) - f32(a[2] * e1[1])), f32(f32(a[2] * e1[0]) - f32(a[0] * e1[2])),
              f32(f32(a[0] * e1[1]) - f32(a[1] * e1[0]))]
        pe1 = f32(f32(f32(p[0] * e1[0]) + f32(p[1] * e1[1])) + f32(p[2] * e1[2]))
        pe2 = f32(f32(f32(p[0] * e2[0]) + f32(p[1] * e2[1])) + f32(p[2] * e2[2]))
        th = f32(f32(math.atan2(float(pe2), float(pe1))) - f32(sp["rot"]))
        if th < f32(-3.14159265):
            th = f32(th + f32(6.28318530))
        if th > f32(3.14159265):
            th = f32(th - f32(6.28318530))
        return int(math.floor(f32(f32(th + f32(3.14159265)) / f32(2.09439510)))) % 3 == sp["idx"]
    return True


def sector_ok(i, j, k, n, pos, splits, h):
    if splits is None or splits[n]["type"] <= 1:
        return True
    d = [f32(f32(f32(c) - f32(pos[n][q])) * h) for q, c in enumerate((i, j, k))]
    r = f32(math.sqrt(f32(f32(f32(d[0] * d[0]) + f32(d[1] * d[1])) + f32(d[2] * d[2]))))
    return in_split(d, r, splits[n])


def evolve(lab, U, W, S, dt_w, curv_reg, groups, pos, splits, h):
    """One pass: snapshot labels in, (labels', W') out, interior cells only."""
    NN = S - 1
    out, Wn = lab.copy(), W.copy()
    L3, U3 = lab.reshape(S, S, S), U.reshape(S, S, S)
    for i in range(1, NN):
        for j in range(1, NN):
            for k in range(1, NN):
                my = int(L3[i, j, k])
                rho_me = f32(U3[i, j, k] * U3[i, j, k])
                best, best_rho, cnt = my, f32(0), f32(0)
                for (a, b, c) in ((i + 1, j, k), (i - 1, j, k), (i, j + 1, k), (i, j - 1, k), (i, j, k + 1),
                                  (i, j, k - 1)):
                    if int(L3[a, b, c]) == my:
                        cnt = f32(cnt + f32(1))
                    else:
                        r = f32(U3[a, b, c] * U3[a, b, c])
                        if r > best_rho:
                            best_rho, best = r, int(L3[a, b, c])
                idx = (i * S + j) * S + k
                w = f32(W[idx])
                if cnt >= 6:
                    Wn[idx] = max(w, f32(1))
                    continue
                if any(my in g and best in g for g in groups):
                    Wn[idx] = max(w, f32(0.5))
                    continue
                den = f32(rho_me + best_rho)
                vel = f32(0) if den < f32(1e-20) else f32(f32(rho_me - best_rho) / den)
                w = f32(w + f32(dt_w * vel))
                w = f32(w + f32(curv_reg * f32(f32(cnt - f32(3)) / f32(3))))
                new = my
                if w < 0:
                    new, w = best, f32(0.1)
                my_ok = sector_ok(i, j, k, my, pos, splits, h)
                if not sector_ok(i, j, k, new, pos, splits, h):
                    new, w = my, max(w, f32(0.1))
                    if not my_ok and best != my and sector_ok(i, j, k, best, pos, splits, h):
                        new, w = best, f32(0.1)
                elif not my_ok and new == my:
                    if best != my and sector_ok(i, j, k, best, pos, splits, h):
                        new, w = best, f32(0.1)
                Wn[idx], out[idx] = w, new
    return out, Wn


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_c_restatement_matches_the_python_one(seed):
    rng = np.random.default_rng(seed)
    S, nA, h = 11, 4, f32(0.4)
    pos = [(int(x), int(y), int(z)) for x, y, z in rng.integers(2, 9, (nA, 3))]
    lab = rng.integers(0, nA, S ** 3).astype(np.uint32)
    U = rng.random(S ** 3).astype(np.float32)
    U[rng.random(S ** 3) < 0.05] = 0  # some zero-density pairs (denominator below 1e-20)
    W = (rng.random(S ** 3) * 1.2 - 0.1).astype(np.float32)
    groups = [[0, 2]] if seed != 1 else [[1, 3], [0, 1]]
    splits = [{"type": 3, "idx": seed % 3, "axis": (0.2, 1.0, 0.4), "rot": 0.3},
              {"type": 2, "idx": 1, "axis": (1.0, -0.5, 0.0), "rot": 0.0},
              {"type": 0, "idx": 0, "axis": (0.0, 0.0, 1.0), "rot": 0.0},
              {"type": 2, "idx": 0, "axis": (0.0, 0.3, 1.0), "rot": 0.0}]
    want_lab, want_W = evolve(lab, U, W, S, f32(0.5), f32(0.15), groups, pos, splits, h)
    rows = [{"i": p[0], "j": p[1], "k": p[2], "Z": 1.0} for p in pos]
    d = orc.MoleculeJsDriver(S - 1, float(h) * (S - 1), rows, locked_groups=groups, splits=splits)
    got_lab, got_W = np.zeros_like(lab), W.copy()
    orc.O().mj_evolve_boundary(lab, got_lab, U, got_W, S, f32(0.5), f32(0.15), d.lock.ctypes.data,
                               orc.C.addressof(d.atoms), d._splits_ptr(), d.h)
    interior = np.zeros((S, S, S), bool)
    interior[1:-1, 1:-1, 1:-1] = True
    interior = interior.reshape(-1)
    assert np.array_equal(got_lab[interior], want_lab[interior])
    assert np.array_equal(got_W.view(np.uint32), want_W.view(np.uint32))
    assert (want_lab[interior] != lab[interior]).any()  # some cells flipped
