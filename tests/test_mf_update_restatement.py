"""A second, pure-Python restatement of mol_fast.js's update shader (mol_fast.js:134-351), written
from the WGSL text independently of oracle/rq_oracle.c and compared bit for bit with the C
restatement on small random grids (CPU): the competition term, the w front, the r_c cusps (every
atom's in the frozen-core form; the orbital's own, the r_out confinement and the hemi / third /
tetra / hemi_third sectors in SHELL_MODE), the Hartree-other term with split-group sharing, the
Thomas-Fermi, tilt, Pauli and field terms, the w-weighted Laplacian of u and the per-electron
Poisson update.  WGSL leaves dot, normalize and atan2 accuracy to the implementation; both
restatements take dot as x0*y0 + x1*y1 + x2*y2, normalize as v / sqrt(dot(v, v)) and atan2 in double
rounded once.  The page's split_rot (set by no page) is 0 on every side.  The GPU kernel is
compared with the C restatement in test_gpu_mol_fast.py."""
import math

import numpy as np

import oracle as orc

f32 = np.float32


def dot3(a, v):
    return f32(f32(f32(a[0] * v[0]) + f32(a[1] * v[1])) + f32(a[2] * v[2]))


def third_sector(ax, rel):
    d = dot3(ax, rel)
    pp = [f32(rel[c] - f32(d * ax[c])) for c in range(3)]
    e1 = [ax[1], f32(-ax[0]), f32(0)] if abs(ax[2]) < f32(0.9) else [f32(0), ax[2], f32(-ax[1])]
    L = f32(math.sqrt(dot3(e1, e1)))
    e1 = [f32(x / L) for x in e1]
    e2 = [f32(f32(ax[1] * e1[2]) - f32(ax[2] * e1[1])), f32(f32(ax[2] * e1[0]) - f32(ax[0] * e1[2])),
          f32(f32(ax[0] * e1[1]) - f32(ax[1] * e1[0]))]
    th = f32(f32(math.atan2(float(dot3(e2, pp)), float(dot3(e1, pp)))) - f32(0))
    if th < f32(-3.141592653589793):
        th = f32(th + f32(6.283185307179586))
    if th > f32(3.141592653589793):
        th = f32(th - f32(6.283185307179586))
    return int(math.floor(f32(f32(th + f32(3.141592653589793)) / f32(2.094395102393195)))) % 3


def in_sector(t, sidx, ax, rel, r_m):
    if t == 2:
        d = dot3(ax, rel)
        return d < 0 if sidx == 0 else d >= 0
    if t == 3:
        return third_sector(ax, rel) == sidx
    if t == 4:
        if r_m > f32(1e-6):
            u = [f32(x / r_m) for x in rel]
            best, bd = 0, dot3([f32(1), f32(1), f32(1)], u)
            for q, v in enumerate(([1, -1, -1], [-1, 1, -1], [-1, -1, 1]), start=1):
                dq = dot3([f32(x) for x in v], u)
                if dq > bd:
                    best, bd = q, dq
            return best == sidx
        return True
    if t == 5:
        d = dot3(ax, rel)
        if sidx == 0:
            return d >= 0
        return False if d >= 0 else third_sector(ax, rel) == sidx - 1
    return True


def cusp(r, rc, h):
    edge = f32(rc - f32(f32(3) * h))
    t = min(max(f32(f32(r - edge) / f32(rc - edge)), f32(0)), f32(1))
    return f32(f32(t * t) * f32(f32(3) - f32(f32(2) * t)))


def restated(p, Ui, Wi, Pi, K):
    NN, S, n = p.NN, p.S, p.n
    S2, S3 = S * S, S ** 3
    h, inv_h, inv_h2, dt, half_d = f32(p.h), f32(p.inv_h), f32(p.inv_h2), f32(p.dt), f32(p.half_d)
    two_pi, alpha, beta, fx, kcm = f32(p.two_pi), f32(p.alpha_tf), f32(p.beta), f32(p.field_x), f32(p.kc_multi)
    atoms = [[f32(v) for v in p.atoms[a]] for a in range(n)]
    rcs = [[f32(v) for v in p.rcs[a]] for a in range(n)]
    axes = [[f32(v) for v in p.ax[a][:3]] for a in range(n)]
    n2 = f32(p.N2)
    Uo, Wo, Po = (np.zeros(n * S3, np.float32) for _ in range(3))
    for i in range(1, NN):
        for j in range(1, NN):
            for k in range(1, NN):
                idx = (i * S + j) * S + k
                for m in range(n):
                    o = m * S3
                    uc = Ui[o + idx]
                    umax = f32(0)
                    for q in range(n):
                        if q != m and Ui[q * S3 + idx] > umax:
                            umax = Ui[q * S3 + idx]
                    cm = f32(uc - umax)
                    wc = Wi[o + idx]
                    wn = [Wi[o + idx + a] for a in (S2, -S2, S, -S, 1, -1)]
                    s = wn[0]
                    for v in wn[1:]:
                        s = f32(s + v)
                    lw = f32(f32(s - f32(f32(6) * wc)) * inv_h2)
                    g = [f32(f32(wn[2 * c] - wn[2 * c + 1]) * inv_h) for c in range(3)]
                    nw = f32(f32(wc + f32(f32(f32(f32(0.05) * dt) * abs(cm)) * lw))
                             + f32(f32(f32(f32(1) * dt) * cm) * f32(math.sqrt(dot3(g, g)))))
                    nw = min(max(nw, f32(0)), f32(1))
                    if p.shell_mode:
                        rel = [f32(f32(c) - atoms[m][q]) for q, c in enumerate((i, j, k))]
                        r_m = f32(f32(math.sqrt(dot3(rel, rel))) * h)
                        rc_m, ro_m = rcs[m][0], f32(f32(p.r_out[m]) * f32(p.R_out))
                        if rc_m > 0 and r_m < rc_m:
                            nw = min(nw, cusp(r_m, rc_m, h))
                        if ro_m > 0 and r_m > ro_m:
                            nw = nw if r_m <= f32(ro_m + h) else f32(0)
                        if p.split_type[m] != 0 and p.split_fix[m] == 1:
                            if not in_sector(p.split_type[m], p.split_idx[m], axes[m], rel, r_m):
                                nw = f32(0)
                    else:
                        for a in range(n):
                            d = [f32(f32(c) - atoms[a][q]) for q, c in enumerate((i, j, k))]
                            r = f32(f32(math.sqrt(dot3(d, d))) * h)
                            if rcs[a][0] > 0 and r < rcs[a][0]:
                                nw = min(nw, cusp(r, rcs[a][0], h))
                    Wo[o + idx] = nw
                    ptot, pgrp = f32(0), f32(0)
                    for q in range(n):
                        ptot = f32(ptot + Pi[q * S3 + idx])
                        if p.split_group[q] == p.split_group[m]:
                            pgrp = f32(pgrp + Pi[q * S3 + idx])
                    self_n = rcs[m][1]
                    fm = (f32(0) if p.full_self > 0.5 else f32(f32(1) / self_n)) if self_n > 1 else f32(1)
                    v_other = f32(f32(2) * f32(ptot - f32(fm * pgrp)))
                    rho_m = f32(uc * uc)
                    v_tf = (f32(alpha * f32(math.pow(float(max(rho_m, f32(1e-20))), float(f32(0.6666667)))))
                            if self_n > 1 and alpha > 0 else f32(0))
                    x_au = f32(f32(f32(i) - n2) * h)
                    y_au = f32(f32(f32(j) - n2) * h)
                    v_tilt = f32(f32(-rcs[m][2] * x_au) - f32(rcs[m][3] * y_au))
                    rho_o = f32(0)
                    for q in range(n):
                        if q != m:
                            rho_o = f32(rho_o + f32(Ui[q * S3 + idx] * Ui[q * S3 + idx]))
                    hd = f32(half_d * (kcm if self_n > 1 else f32(1)))
                    un6 = [Ui[o + idx + a] for a in (S2, -S2, S, -S, 1, -1)]
                    unew = uc
                    for c in range(3):
                        xp = f32(f32(f32(un6[2 * c] - uc) * f32(wn[2 * c] + nw)) * f32(0.5))
                        xm = f32(f32(f32(uc - un6[2 * c + 1]) * f32(nw + wn[2 * c + 1])) * f32(0.5))
                        unew = f32(unew + f32(hd * f32(xp - xm)))
                    pot = f32(f32(f32(f32(f32(K[idx] - v_other) - v_tf) - v_tilt) - f32(beta * rho_o)) - f32(fx * x_au))
                    Uo[o + idx] = f32(unew + f32(f32(f32(dt * pot) * uc) * wc))
                    pc = Pi[o + idx]
                    ps = Pi[o + idx + S2]
                    for a in (-S2, S, -S, 1, -1):
                        ps = f32(ps + Pi[o + idx + a])
                    Po[o + idx] = f32(f32(pc + f32(f32(dt * f32(ps - f32(f32(6) * pc))) * inv_h2))
                                      + f32(f32(f32(two_pi * dt) * uc) * uc))
    return Uo, Wo, Po


def compare(d, seed):
    p = d.p
    S3 = p.S ** 3
    rng = np.random.default_rng(seed)
    Ui = rng.random(p.n * S3).astype(np.float32)
    Wi = rng.random(p.n * S3).astype(np.float32)
    Pi = (rng.random(p.n * S3) * 0.5).astype(np.float32)
    K = (rng.random(S3) * 3).astype(np.float32)
    got = [np.zeros(p.n * S3, np.float32) for _ in range(3)]
    orc.O().mf_update(orc.C.addressof(p), Ui, Wi, Pi, K, *got)
    want = restated(p, Ui, Wi, Pi, K)
    interior = np.zeros((p.S,) * 3, bool)
    interior[1:-1, 1:-1, 1:-1] = True
    sel = np.tile(interior.reshape(-1), p.n)
    for name, g, w in zip("UWP", got, want):
        assert np.array_equal(g[sel].view(np.uint32), w[sel].view(np.uint32)), name
    return want


def test_frozen_core_update_matches_a_python_restatement():
    nuc = [{"i": 4, "j": 5, "k": 5, "Z": 3, "rc": 0.6, "z_init": 2.5, "tilt_y": 0.01},
           {"i": 7, "j": 5.5, "k": 6, "Z": 1, "tilt_x": -0.02},
           {"i": 3.25, "j": 6, "k": 5, "Z": 0, "z_init": 1.2}]
    d = orc.MolFastDriver(nuc, NN=10, screen=4.0, norm_targets=[2, 1, 1], kc_multi=1.5, beta_pauli=0.05,
                          field_x=0.01, alpha_tf=0.2)
    compare(d, 8)


def test_shell_mode_update_matches_a_python_restatement():
    """SHELL_MODE: own r_c cusp, r_out confinement, hemi / third / tetra / hemi_third sectors and
    split siblings sharing their Hartree subtraction."""
    nuc = [{"i": 6, "j": 6, "k": 6, "Z": 2, "rc": 0.5, "split": "hemi", "split_idx": 0, "split_axis": [1, 1, 0]},
           {"i": 6, "j": 6, "k": 6, "Z": 2, "rc": 0.5, "split": "hemi", "split_idx": 1, "split_axis": [1, 1, 0]},
           {"i": 6, "j": 6, "k": 6, "Z": 1, "r_out": 1.0, "split": "third", "split_idx": 2, "split_axis": [0, 0, 1]},
           {"i": 6, "j": 6, "k": 6, "Z": 1, "split": "tetra", "split_idx": 1},
           {"i": 8, "j": 6, "k": 6, "Z": 1, "split": "hemi_third", "split_idx": 2, "split_axis": [0.3, 0.2, 1.0]},
           {"i": 4, "j": 7, "k": 6, "Z": 1, "split": "hemi_third", "split_idx": 0, "split_fix": False}]
    d = orc.MolFastDriver(nuc, NN=12, screen=3.6, shell_mode=True)
    Uo, Wo, Po = compare(d, 9)
    S3 = d.p.S ** 3
    assert (Wo[2 * S3:3 * S3] == 0).sum() > (Wo[5 * S3:] == 0).sum()  # sectors and r_out zero w cells


def test_reduction_trees_match_a_python_restatement():
    """reduceWGSL + finalizeWGSL (mol_fast.js:353-472): per cell the n norms and T (kinetic where
    w > 0.1, Thomas-Fermi, tilt), V_eK, V_ee (P_tot - f_m P_m) and the dipole; each 128-cell
    workgroup folds pairwise, one workgroup adds the partials in strides of 128 and folds again."""
    nuc = [{"i": 4, "j": 5, "k": 5, "Z": 3, "rc": 0.6, "z_init": 2.5, "tilt_y": 0.01},
           {"i": 7, "j": 5.5, "k": 6, "Z": 1, "tilt_x": -0.02},
           {"i": 3.25, "j": 6, "k": 5, "Z": 0, "z_init": 1.2}]
    d = orc.MolFastDriver(nuc, NN=12, screen=4.8, norm_targets=[2, 1, 1], kc_multi=1.5, alpha_tf=0.2)
    p = d.p
    n, S, NN = p.n, p.S, p.NN
    S2, S3 = S * S, S ** 3
    rng = np.random.default_rng(12)
    U = rng.random(n * S3).astype(np.float32)
    W = rng.random(n * S3).astype(np.float32)
    P = (rng.random(n * S3) * 0.5).astype(np.float32)
    K = (rng.random(S3) * 3).astype(np.float32)
    got = np.zeros(n + 6, np.float32)
    orc.O().mf_reduce(orc.C.addressof(p), U, W, P, K, got)
    h, h3, n2 = f32(p.h), f32(p.h3), f32(p.N2)
    kc, kcm, alpha = f32(p.kc), f32(p.kc_multi), f32(p.alpha_tf)
    rcs = [[f32(v) for v in p.rcs[a]] for a in range(n)]
    NR, NM = n + 6, NN - 1
    tot = NM ** 3
    nwg = -(-tot // 128)
    parts = []
    for w in range(nwg):
        sn = [[f32(0)] * NR for _ in range(128)]
        for lid in range(128):
            cell = w * 128 + lid
            if cell >= tot:
                continue
            k, j, i = cell % NM + 1, (cell // NM) % NM + 1, cell // (NM * NM) + 1
            idx = (i * S + j) * S + k
            T = VeK = Vee = dx = dy = dz = f32(0)
            xc, yc, zc = (f32(f32(f32(c) - n2) * h) for c in (i, j, k))
            ptot = f32(0)
            for q in range(n):
                ptot = f32(ptot + P[q * S3 + idx])
            for m in range(n):
                o = m * S3
                v = U[o + idx]
                sn[lid][m] = f32(f32(v * v) * h3)
                self_n = rcs[m][1]
                if W[o + idx] > f32(0.1):
                    a_, b_, c_ = (f32(U[o + idx + s] - v) for s in (S2, S, 1))
                    km = kcm if self_n > 1 else f32(1)
                    T = f32(T + f32(f32(f32(km * kc) * f32(f32(f32(a_ * a_) + f32(b_ * b_)) + f32(c_ * c_))) * h))
                VeK = f32(VeK - f32(f32(f32(K[idx] * v) * v) * h3))
                rho_cell = f32(f32(v * v) * h3)
                dx, dy, dz = f32(dx - f32(rho_cell * xc)), f32(dy - f32(rho_cell * yc)), f32(dz - f32(rho_cell * zc))
                fm = f32(f32(1) / self_n) if self_n > 1 else f32(1)
                Vee = f32(Vee + f32(f32(f32(f32(ptot - f32(fm * P[o + idx])) * v) * v) * h3))
                if self_n > 1 and alpha > 0:
                    rho_m = f32(v * v)
                    pw = f32(math.pow(float(max(rho_m, f32(1e-20))), float(f32(1.6666667))))
                    T = f32(T + f32(f32(f32(f32(0.6) * alpha) * pw) * h3))
                tilt = rcs[m][3]
                if tilt != 0:
                    T = f32(T + f32(f32(f32(f32(f32(-tilt) * yc) * v) * v) * h3))
            sn[lid][n:] = [T, VeK, Vee, dx, dy, dz]
        s = 64
        while s > 0:
            for lid in range(s):
                sn[lid] = [f32(x + y) for x, y in zip(sn[lid], sn[lid + s])]
            s //= 2
        parts.append(sn[0])
    wg = [[f32(0)] * NR for _ in range(128)]
    for lid in range(128):
        for w in range(lid, nwg, 128):
            wg[lid] = [f32(x + y) for x, y in zip(wg[lid], parts[w])]
    s = 64
    while s > 0:
        for lid in range(s):
            wg[lid] = [f32(x + y) for x, y in zip(wg[lid], wg[lid + s])]
        s //= 2
    assert np.array_equal(np.array(wg[0], np.float32).view(np.uint32), got.view(np.uint32))
