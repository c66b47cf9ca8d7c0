"""Second, pure-Python restatements of molecule.js's per-step shaders, written from the WGSL text
independently of oracle/rq_oracle.c: updateU with the r_c exclusion and a bare nucleus
(molecule.js:228-343, W_CUTOFF = 0 so mix(uc, u_raw, 1) = u_raw), the weighted Jacobi sweep with its
literal 0.3333 (:723-749), the fixed-point norms and their decoding (:911-946) and normalize
(:1077-1105).  Each is compared bit for bit with the C restatement on a small random grid (CPU);
the GPU kernels are compared with the C restatement in test_gpu_mj.py."""
import numpy as np

import oracle as orc

f32 = np.float32
S = 9
ROWS = [{"i": 3, "j": 4, "k": 4, "Z": 2.0, "Z_nuc": 2.0, "rc": 0.5},
        {"i": 6, "j": 4, "k": 5, "Z": 1.0, "Z_nuc": 1.0, "rc": 0.0},
        {"i": 4, "j": 6, "k": 3, "Z": 0.0, "Z_nuc": 1.0, "rc": 0.35}]  # a bare nucleus
H = f32(0.4)


def state(seed):
    rng = np.random.default_rng(seed)
    n = S ** 3
    return (rng.random(n).astype(np.float32), rng.integers(0, 2, n).astype(np.uint32),
            np.abs(rng.normal(size=n)).astype(np.float32), rng.normal(size=n).astype(np.float32) * f32(0.3))


def dist(c, a):
    d = [f32(f32(f32(x) - f32(a[q])) * H) for q, x in zip("ijk", c)]
    return f32(np.sqrt(f32(f32(f32(d[0] * d[0]) + f32(d[1] * d[1])) + f32(d[2] * d[2]))))


def inside_rc(c, lbl, has_bare):
    """updateU's isInsideRc (molecule.js:246-259), the bare-nuclei loop compiled in when present."""
    a = ROWS[lbl]
    if a["rc"] > 0 and dist(c, a) < f32(a["rc"]):
        return True
    if has_bare:
        for b in ROWS:
            if b["Z"] <= 0 and b["Z_nuc"] > 0 and b["rc"] > 0 and dist(c, b) < f32(b["rc"]):
                return True
    return False


def interior():
    for i in range(1, S - 1):
        for j in range(1, S - 1):
            for k in range(1, S - 1):
                yield i, j, k, (i * S + j) * S + k


def test_update_matches_a_python_restatement():
    U, label, K, Pother = state(1)
    half_d, dt = f32(0.06), f32(0.12 * 0.16)
    got = np.zeros_like(U)
    atoms = orc.mj_atoms(ROWS)
    orc.O().mj_update(U, got, K, label, Pother, orc.C.addressof(atoms), len(ROWS), 1, S, H, half_d, dt)
    steps = {(1, 0, 0): S * S, (-1, 0, 0): -S * S, (0, 1, 0): S, (0, -1, 0): -S, (0, 0, 1): 1, (0, 0, -1): -1}
    excluded = 0
    for i, j, k, idx in interior():
        my = int(label[idx])
        if inside_rc((i, j, k), my, True):
            want = f32(0)
            excluded += 1
        else:
            uc = U[idx]
            acc = None
            for (di, dj, dk), off in steps.items():
                ln = int(label[idx + off])
                v = U[idx + off] if ln == my and not inside_rc((i + di, j + dj, k + dk), ln, True) else uc
                acc = v if acc is None else f32(acc + v)
            lap = f32(acc - f32(f32(6) * uc))
            want = f32(f32(uc + f32(half_d * lap)) + f32(f32(dt * f32(K[idx] - f32(f32(2) * Pother[idx]))) * uc))
        assert got[idx].view(np.uint32) == want.view(np.uint32), (i, j, k)
    assert excluded > 0


def test_weighted_jacobi_matches_a_python_restatement():
    U, _, _, P = state(2)
    rho = np.zeros_like(U)
    orc.O().mj_rho(U, rho, S)
    got = np.zeros_like(P)
    h2, two_pi = f32(0.16), f32(2 * np.pi)
    orc.O().mj_jacobi(P, got, rho, S, h2, two_pi)
    for i, j, k, idx in interior():
        s = P[idx + S * S]
        for off in (-S * S, S, -S, 1, -1):
            s = f32(s + P[idx + off])
        rhs = f32(f32(h2 * two_pi) * f32(U[idx] * U[idx]))
        want = f32(f32(f32(0.3333) * P[idx]) + f32(f32(s + rhs) / f32(9)))
        assert got[idx].view(np.uint32) == want.view(np.uint32), (i, j, k)


def test_fixed_point_norms_and_normalize_match_a_python_restatement():
    U, label, _, _ = state(3)
    h3 = f32(0.064)
    acc = np.zeros(len(ROWS), np.uint32)
    nf = np.zeros(len(ROWS), np.float32)
    orc.O().mj_norms_fixed(U, label, S, h3, len(ROWS), acc, nf)
    want = [0, 0, 0]
    for *_, idx in interior():
        want[int(label[idx])] = (want[int(label[idx])] + int(f32(f32(f32(U[idx] * U[idx]) * h3) * f32(16777216)))) % 2 ** 32
    assert list(acc) == want
    dec = [f32(f32(a) * f32(1 / 16777216)) for a in want]
    assert np.array_equal(nf.view(np.uint32), np.array(dec, np.float32).view(np.uint32))
    V = U.copy()
    orc.O().mj_normalize(V, nf, label, orc.C.addressof(orc.mj_atoms(ROWS)), S)
    for *_, idx in interior():
        l = int(label[idx])
        n, Z = dec[l], f32(ROWS[l]["Z"])
        w = f32(U[idx] * f32(np.sqrt(f32(Z / n)))) if (n > 0 and Z > 0) else U[idx]
        assert V[idx].view(np.uint32) == w.view(np.uint32)


def test_two_level_correction_matches_a_python_restatement():
    """The V-cycle pieces (molecule.js:772-909): residual r = -2 pi rho - lap P, the 27-point
    full-weighting restriction (weights 8/4/2/1, times 1/64), the coarse weighted Jacobi with
    h_c^2 = 4 h^2 and 0.3333, and the trilinear prolongation added at half weight."""
    rng = np.random.default_rng(5)
    NN = S - 1
    NC, SC = NN // 2, NN // 2 + 1
    P = rng.normal(size=S ** 3).astype(np.float32)
    rho = rng.random(S ** 3).astype(np.float32)
    inv_h2, h2, two_pi = f32(1 / 0.16), f32(0.16), f32(2 * np.pi)
    R = np.zeros_like(P)
    orc.O().mj_residual(P, R, rho, S, inv_h2, two_pi)
    for i, j, k, idx in interior():
        s = P[idx + S * S]
        for off in (-S * S, S, -S, 1, -1):
            s = f32(s + P[idx + off])
        lap = f32(f32(s - f32(f32(6) * P[idx])) * inv_h2)
        want = f32(f32(-two_pi * rho[idx]) - lap)
        assert R[idx].view(np.uint32) == want.view(np.uint32)
    fc = np.zeros(SC ** 3, np.float32)
    orc.O().mj_restrict(R, fc, S, SC)
    F3 = R.reshape(S, S, S)
    faces = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    edges = [(1, 1, 0), (1, -1, 0), (-1, 1, 0), (-1, -1, 0), (1, 0, 1), (1, 0, -1), (-1, 0, 1), (-1, 0, -1),
             (0, 1, 1), (0, 1, -1), (0, -1, 1), (0, -1, -1)]
    corners = [(1, 1, 1), (1, 1, -1), (1, -1, 1), (1, -1, -1), (-1, 1, 1), (-1, 1, -1), (-1, -1, 1), (-1, -1, -1)]

    def ssum(fi, fj, fk, offs):
        acc = None
        for a, b, c in offs:
            v = F3[fi + a, fj + b, fk + c]
            acc = v if acc is None else f32(acc + v)
        return acc

    want_c = np.zeros_like(fc)
    for I in range(1, NC):
        for J in range(1, NC):
            for K2 in range(1, NC):
                fi, fj, fk = 2 * I, 2 * J, 2 * K2
                val = f32(f32(8) * F3[fi, fj, fk])
                val = f32(val + f32(f32(4) * ssum(fi, fj, fk, faces)))
                val = f32(val + f32(f32(2) * ssum(fi, fj, fk, edges)))
                val = f32(val + ssum(fi, fj, fk, corners))
                want_c[(I * SC + J) * SC + K2] = f32(val * f32(0.015625))
    assert np.array_equal(fc.view(np.uint32), want_c.view(np.uint32))
    E0 = rng.normal(size=SC ** 3).astype(np.float32)
    E1 = np.zeros_like(E0)
    orc.O().mj_coarse_smooth(E0, E1, fc, SC, h2)
    for I in range(1, NC):
        for J in range(1, NC):
            for K2 in range(1, NC):
                c = (I * SC + J) * SC + K2
                s = E0[c + SC * SC]
                for off in (-SC * SC, SC, -SC, 1, -1):
                    s = f32(s + E0[c + off])
                want = f32(f32(f32(0.3333) * E0[c]) + f32(f32(s + f32(f32(f32(4) * h2) * fc[c])) / f32(9)))
                assert E1[c].view(np.uint32) == want.view(np.uint32)
    Pf = P.copy()
    orc.O().mj_prolong(E1, Pf, S, SC)
    for i, j, k, idx in interior():
        ci, cj, ck = i // 2, j // 2, k // 2
        c1 = [min(x // 2 + (x & 1), NC) for x in (i, j, k)]
        w = [f32(0.5) if (x & 1) else f32(1) for x in (i, j, k)]
        w1 = [f32(f32(1) - x) for x in w]
        corr = f32(0)
        for a in (0, 1):
            for b in (0, 1):
                for c in (0, 1):
                    wa, wb, wc = (w[0] if a == 0 else w1[0]), (w[1] if b == 0 else w1[1]), (w[2] if c == 0 else w1[2])
                    ii, jj, kk = (ci if a == 0 else c1[0]), (cj if b == 0 else c1[1]), (ck if c == 0 else c1[2])
                    corr = f32(corr + f32(f32(f32(wa * wb) * wc) * E1[(ii * SC + jj) * SC + kk]))
        want = f32(P[idx] + f32(f32(0.5) * corr))
        assert Pf[idx].view(np.uint32) == want.view(np.uint32), (i, j, k)


def test_self_interaction_and_direct_path_helpers_match_a_python_restatement():
    """computeRhoSelf / computeRhoOther (molecule.js:572-619), initPdirect (:621-662),
    copyPotherForLabel (:665-692) and subtractPself (:694-720, fraction 1/Z for Z > 1)."""
    U, label, _, Pother = state(4)
    label = (label + (np.arange(S ** 3) % 3 == 0)).astype(np.uint32)  # labels 0, 1, 2
    m = 1
    rs, ro = np.full_like(U, 7.0), np.full_like(U, 7.0)
    orc.O().mj_rho_self(U, label, m, rs, S)
    orc.O().mj_rho_other(U, label, m, ro, S)
    Pm = np.random.default_rng(6).normal(size=S ** 3).astype(np.float32)
    cp, sub = Pother.copy(), Pother.copy()
    orc.O().mj_copy_for_label(Pm, cp, label, m, S)
    Z = f32(2.0)
    orc.O().mj_sub_self(Pm, sub, label, m, Z, S)
    atoms = orc.mj_atoms(ROWS)
    pd, po = np.zeros_like(U), Pother.copy()
    orc.O().mj_init_pdirect(orc.C.addressof(atoms), len(ROWS), 0, pd, po, S, H, f32(H * H))
    h2 = f32(H * H)
    for i, j, k, idx in interior():
        u2 = f32(U[idx] * U[idx])
        own = int(label[idx]) == m
        assert rs[idx].view(np.uint32) == (u2 if own else f32(0)).view(np.uint32)
        assert ro[idx].view(np.uint32) == (f32(0) if own else u2).view(np.uint32)
        assert cp[idx].view(np.uint32) == (Pm[idx] if own else Pother[idx]).view(np.uint32)
        want = f32(Pother[idx] - f32(Pm[idx] * f32(f32(1) / Z))) if own else Pother[idx]
        assert sub[idx].view(np.uint32) == want.view(np.uint32)
        xi, yj, zk = (f32(f32(c) * H) for c in (i, j, k))
        val = f32(0)
        for q, a in enumerate(ROWS):
            if f32(a["Z"]) <= 0 or q == 0:
                continue
            dx, dy, dz = (f32(x - f32(f32(a[c]) * H)) for x, c in zip((xi, yj, zk), "ijk"))
            r = f32(np.sqrt(f32(f32(f32(f32(dx * dx) + f32(dy * dy)) + f32(dz * dz)) + h2)))
            val = f32(val + f32(f32(0.5) / r))
        assert pd[idx].view(np.uint32) == val.view(np.uint32)
        assert po[idx].view(np.uint32) == f32(Pother[idx] + val).view(np.uint32)
