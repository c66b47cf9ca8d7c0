"""A second, pure-Python restatement of mol_fast.js's update shader in its frozen-core form
(SHELL_MODE off, mol_fast.js:134-351: the competition term, the w front with the r_c cusps of every
atom, the Hartree-other, Thomas-Fermi, tilt, Pauli and field terms, the w-weighted Laplacian of u,
the per-electron Poisson update), written from the WGSL text independently of oracle/rq_oracle.c and
compared bit for bit with the C restatement on a small random grid (CPU).  The GPU kernel is
compared with the C restatement in test_gpu_mol_fast.py."""
import math

import numpy as np

import oracle as orc

f32 = np.float32
NUC = [{"i": 4, "j": 5, "k": 5, "Z": 3, "rc": 0.6, "z_init": 2.5, "tilt_y": 0.01},
       {"i": 7, "j": 5.5, "k": 6, "Z": 1, "tilt_x": -0.02},
       {"i": 3.25, "j": 6, "k": 5, "Z": 0, "z_init": 1.2}]


def test_frozen_core_update_matches_a_python_restatement():
    NN = 10
    d = orc.MolFastDriver(NUC, NN=NN, screen=4.0, norm_targets=[2, 1, 1], kc_multi=1.5, beta_pauli=0.05,
                          field_x=0.01, alpha_tf=0.2)
    p = d.p
    S, n = NN + 1, len(NUC)
    S2, S3 = S * S, S ** 3
    rng = np.random.default_rng(8)
    Ui = rng.random(n * S3).astype(np.float32)
    Wi = rng.random(n * S3).astype(np.float32)
    Pi = (rng.random(n * S3) * 0.5).astype(np.float32)
    K = (rng.random(S3) * 3).astype(np.float32)
    Uo, Wo, Po = (np.zeros(n * S3, np.float32) for _ in range(3))
    orc.O().mf_update(orc.C.addressof(p), Ui, Wi, Pi, K, Uo, Wo, Po)
    h, inv_h, inv_h2, dt, half_d = f32(p.h), f32(p.inv_h), f32(p.inv_h2), f32(p.dt), f32(p.half_d)
    two_pi, alpha, beta, fx, kcm = f32(p.two_pi), f32(p.alpha_tf), f32(p.beta), f32(p.field_x), f32(p.kc_multi)
    atoms = [[f32(v) for v in p.atoms[a]] for a in range(n)]
    rcs = [[f32(v) for v in p.rcs[a]] for a in range(n)]
    n2 = f32(p.N2)
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
                             + f32(f32(f32(f32(1) * dt) * cm)
                                   * f32(math.sqrt(f32(f32(f32(g[0] * g[0]) + f32(g[1] * g[1])) + f32(g[2] * g[2]))))))
                    nw = min(max(nw, f32(0)), f32(1))
                    for a in range(n):  # frozen core: every atom's rc
                        dx, dy, dz = (f32(f32(c) - atoms[a][q]) for q, c in enumerate((i, j, k)))
                        r = f32(f32(math.sqrt(f32(f32(f32(dx * dx) + f32(dy * dy)) + f32(dz * dz)))) * h)
                        rc = rcs[a][0]
                        if rc > 0 and r < rc:
                            edge = f32(rc - f32(f32(3) * h))
                            t = min(max(f32(f32(r - edge) / f32(rc - edge)), f32(0)), f32(1))
                            nw = min(nw, f32(f32(t * t) * f32(f32(3) - f32(f32(2) * t))))
                    assert Wo[o + idx].view(np.uint32) == nw.view(np.uint32), ("w", i, j, k, m)
                    ptot, pgrp = f32(0), f32(0)
                    for q in range(n):
                        ptot = f32(ptot + Pi[q * S3 + idx])
                        if q == m:
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
                            un = Ui[q * S3 + idx]
                            rho_o = f32(rho_o + f32(un * un))
                    v_pauli = f32(beta * rho_o)
                    hd = f32(half_d * (kcm if self_n > 1 else f32(1)))
                    un6 = [Ui[o + idx + a] for a in (S2, -S2, S, -S, 1, -1)]
                    unew = uc
                    for c in range(3):
                        xp = f32(f32(f32(un6[2 * c] - uc) * f32(wn[2 * c] + nw)) * f32(0.5))
                        xm = f32(f32(f32(uc - un6[2 * c + 1]) * f32(nw + wn[2 * c + 1])) * f32(0.5))
                        unew = f32(unew + f32(hd * f32(xp - xm)))
                    pot = f32(f32(f32(f32(f32(K[idx] - v_other) - v_tf) - v_tilt) - v_pauli) - f32(fx * x_au))
                    unew = f32(unew + f32(f32(f32(dt * pot) * uc) * wc))
                    assert Uo[o + idx].view(np.uint32) == unew.view(np.uint32), ("u", i, j, k, m)
                    pc = Pi[o + idx]
                    ps = Pi[o + idx + S2]
                    for a in (-S2, S, -S, 1, -1):
                        ps = f32(ps + Pi[o + idx + a])
                    pn = f32(f32(pc + f32(f32(dt * f32(ps - f32(f32(6) * pc))) * inv_h2))
                             + f32(f32(f32(two_pi * dt) * uc) * uc))
                    assert Po[o + idx].view(np.uint32) == pn.view(np.uint32), ("P", i, j, k, m)
