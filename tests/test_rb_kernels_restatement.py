"""Second, pure-Python restatements of realqm_rb.js's red-black passes, written from the WGSL text
independently of oracle/rq_oracle.c: the fused front + amplitude pass fusedWU_RB
(realqm_rb.js:256-316, in place; same-colour cells never read each other) and the in-place Poisson
pass updateP_RB (:318-354, with the (n-1)/n self term of a multiply occupied orbital).  Compared
bit for bit with the C restatement on a small random grid (CPU); the GPU kernels are compared
with the C restatement in test_gpu_realqm_rb.py."""
import numpy as np
import pytest

import oracle as orc

f32 = np.float32
S, NN = 9, 8


def params(tgt):
    p = orc.RbParams()
    h = 0.35
    p.NN, p.S, p.N2, p.n = NN, S, NN // 2, len(tgt)
    p.h, p.h2, p.inv_h, p.inv_h2 = f32(h), f32(h * h), f32(1 / h), f32(1 / (h * h))
    p.dt, p.half_d, p.two_pi, p.h3 = f32(0.1 * h * h), f32(0.05), f32(2 * np.pi), f32(h ** 3)
    for m, t in enumerate(tgt):
        p.tgt[m] = t
    return p


def cells(color):
    for i in range(1, NN):
        for j in range(1, NN):
            for k in range(1, NN):
                if (i + j + k) % 2 == color:
                    yield (i * S + j) * S + k


@pytest.mark.parametrize("color", [0, 1])
def test_fused_front_and_amplitude_pass(color):
    rng = np.random.default_rng(11 + color)
    n, m = 2, 1
    S3 = S ** 3
    U = rng.random(n * S3).astype(np.float32)
    W = (rng.random(n * S3) * 1.5 - 0.2).astype(np.float32)
    un = rng.random(n * S3).astype(np.float32)
    K = np.abs(rng.normal(size=S3)).astype(np.float32)
    P = (rng.random(n * S3) * 0.4).astype(np.float32)
    mask = (rng.random(n * S3) > 0.1).astype(np.float32)
    p = params([1.0, 1.0])
    U1, W1 = U.copy(), W.copy()
    orc.O().rb_wu(orc.C.addressof(p), m, color, U1, W1, un, K, P, mask)
    u, w = U[m * S3:(m + 1) * S3].copy(), W[m * S3:(m + 1) * S3].copy()
    nu, Pm, mk = un[m * S3:], P[m * S3:], mask[m * S3:]
    dt, inv_h, inv_h2, half_d = f32(p.dt), f32(p.inv_h), f32(p.inv_h2), f32(p.half_d)
    for idx in cells(color):
        nb = (S * S, -S * S, S, -S, 1, -1)
        c = f32(f32(0.1) * f32(u[idx] - nu[idx]))
        wc = w[idx]
        s = w[idx + nb[0]]
        for off in nb[1:]:
            s = f32(s + w[idx + off])
        lap_w = f32(s - f32(f32(6) * wc))
        g = [f32(f32(w[idx + a] - w[idx - a]) * inv_h) for a in (S * S, S, 1)]
        grad = f32(np.sqrt(f32(f32(f32(g[0] * g[0]) + f32(g[1] * g[1])) + f32(g[2] * g[2]))))
        w[idx] = f32(f32(wc + f32(f32(f32(f32(f32(0.5) * dt) * abs(c)) * lap_w) * inv_h2))
                     + f32(f32(f32(f32(10) * dt) * c) * grad))
        wc2, uc = w[idx], u[idx]
        fl = []
        for a in (S * S, S, 1):
            fp = f32(f32(f32(u[idx + a] - uc) * f32(w[idx + a] + wc2)) * f32(0.5))
            fm = f32(f32(f32(uc - u[idx - a]) * f32(wc2 + w[idx - a])) * f32(0.5))
            fl.append(f32(fp - fm))
        wlap = f32(f32(fl[0] + fl[1]) + fl[2])
        unew = f32(f32(uc + f32(half_d * wlap)) + f32(f32(f32(dt * f32(K[idx] - f32(f32(2) * Pm[idx]))) * uc) * wc2))
        u[idx] = f32(unew * mk[idx])
        w[idx] = f32(w[idx] * mk[idx])
    assert np.array_equal(U1[m * S3:(m + 1) * S3].view(np.uint32), u.view(np.uint32))
    assert np.array_equal(W1[m * S3:(m + 1) * S3].view(np.uint32), w.view(np.uint32))
    assert np.array_equal(U1[:S3], U[:S3]) and np.array_equal(W1[:S3], W[:S3])  # the other electron untouched


@pytest.mark.parametrize("color,tgt", [(0, 1.0), (1, 2.0)])
def test_poisson_pass(color, tgt):
    rng = np.random.default_rng(21 + color)
    S3 = S ** 3
    P = rng.normal(size=2 * S3).astype(np.float32) * f32(0.3)
    U = rng.random(2 * S3).astype(np.float32)
    rho = (rng.random(S3) * 2).astype(np.float32)
    p = params([1.0, tgt])
    m = 1
    P1 = P.copy()
    orc.O().rb_p(orc.C.addressof(p), m, color, P1, U, rho)
    Pm, us = P[m * S3:(m + 1) * S3].copy(), U[m * S3:]
    dt, inv_h2, two_pi = f32(p.dt), f32(p.inv_h2), f32(p.two_pi)
    sf = f32(f32(1) / f32(tgt)) if f32(tgt) > 1 else f32(1)
    for idx in cells(color):
        s = Pm[idx + S * S]
        for off in (-S * S, S, -S, 1, -1):
            s = f32(s + Pm[idx + off])
        lap = f32(s - f32(f32(6) * Pm[idx]))
        others = max(f32(rho[idx] - f32(f32(sf * us[idx]) * us[idx])), f32(0))
        Pm[idx] = f32(Pm[idx] + f32(dt * f32(f32(lap * inv_h2) + f32(two_pi * others))))
    assert np.array_equal(P1[m * S3:(m + 1) * S3].view(np.uint32), Pm.view(np.uint32))


def test_norm_reduction_and_normalize():
    """reduceNormWGSL + normalizeWGSL (realqm_rb.js:356-427): N_REDUCE_WG = min(256, ceil(cells/128))
    workgroups of 128 threads, each thread striding over the interior cells, the pairwise fold, then
    every normalize thread adds the partials in order and scales u by sqrt(tgt / norm)."""
    rng = np.random.default_rng(31)
    S3 = S ** 3
    U = rng.random(2 * S3).astype(np.float32)
    p = params([1.0, 2.0])
    m = 1
    U1 = U.copy()
    got = orc.O().rb_normalize(orc.C.addressof(p), m, U1)
    h3 = f32(p.h3)
    NM = NN - 1
    tot = NM ** 3
    nwg = min(256, -(-tot // 128))
    u = U[m * S3:(m + 1) * S3]
    parts = []
    for w in range(nwg):
        sd = []
        for lid in range(128):
            acc = f32(0)
            cell = w * 128 + lid
            while cell < tot:
                k, j, i = cell % NM + 1, (cell // NM) % NM + 1, cell // (NM * NM) + 1
                v = u[(i * S + j) * S + k]
                acc = f32(acc + f32(f32(v * v) * h3))
                cell += nwg * 128
            sd.append(acc)
        s = 64
        while s > 0:
            for lid in range(s):
                sd[lid] = f32(sd[lid] + sd[lid + s])
            s //= 2
        parts.append(sd[0])
    norm = f32(0)
    for x in parts:
        norm = f32(norm + x)
    assert np.float32(got).view(np.uint32) == norm.view(np.uint32)
    sc = f32(np.sqrt(f32(f32(2.0) / norm)))
    want = u.copy()
    for i in range(1, NN):
        for j in range(1, NN):
            for k in range(1, NN):
                idx = (i * S + j) * S + k
                want[idx] = f32(u[idx] * sc)
    assert np.array_equal(U1[m * S3:(m + 1) * S3].view(np.uint32), want.view(np.uint32))
