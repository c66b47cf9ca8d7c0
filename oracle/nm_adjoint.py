"""FP64 restatement of the new flavour's adjoint (TEST INFRASTRUCTURE ONLY).

Only tests/ may import this module.  ``gradient(drv, n_steps)`` runs ``n_steps`` of an
``oracle.NewMethodDriver`` (labels frozen) while recording the state every step starts from,
then runs the reverse sweep in numpy and returns the energy readout, the electronic force
-dE/dR on every entry and dE/dK on the grid (which is dE/dv for an external potential).

The forward step (oracle.NewMethodDriver.step) is, on the normalised state,
    [V-cycle]    P <- M P + B f,  f = 2 pi psi^2        (every poisson_interval steps)
    update       psi~ = psi + half_dv L psi + dt (K - 2P) psi     (L: same-label Laplacian)
    [normalise]  psi = c psi~,  c_d = sqrt(Z_d / (h^3 sum_d psi~^2))
and the readout is E = sum_d (Z_d / N_d)(T_d + V_eK,d + 2 h^3 sum_d P rho) - (h^3 / 2 pi) sum P A P
(the P-stationary Hartree form, A = -lap_h).  The reverse sweep applies the
transposes newest step first: normalise^T lam <- c (lam - (h^3/Z) psi <psi, lam>_d); update^T
lam <- A lam with dE/dK += dt psi lam and dE/dP += -2 dt psi lam; V-cycle^T by transposing every
red-black colour, the residual, full weighting (its transpose is the prolongation / 8), the
trilinear prolongation (its transpose is 8 x full weighting) and the coarsest sweeps in reverse
order (orc_nm_vcycle, oracle/rq_oracle.c, is the forward).  The gather is
F_a = sum_i dE/dK_i dK_a/dr (x_i - R_a) / r with K_a = Z_a erf(r / (sqrt 2 sigma)) / r.
"""
from __future__ import annotations

import math

import numpy as np

import oracle as orc

_SH = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]


def _nb(X, d):
    """The neighbour in direction d of every interior point (interior-shaped view)."""
    n = X.shape[0]
    a, b, c = d
    return X[1 + a:n - 1 + a, 1 + b:n - 1 + b, 1 + c:n - 1 + c]


def _in(X):
    return X[1:-1, 1:-1, 1:-1]


def _same_label_lap(X, L):
    """sum over same-label neighbours of (X_nb - X) at interior points (Dirichlet faces: X = 0 there)."""
    c, lc = _in(X), _in(L)
    out = np.zeros_like(c)
    for d in _SH:
        out += np.where(_nb(L, d) == lc, _nb(X, d) - c, 0.0)
    return out


def _colors(S):
    g = np.indices((S, S, S)).sum(0) & 1
    return _in(g)


def _adj_color(mu, muf, h2, color, par):
    """One red-black colour transposed: at colour points muf += h2/6 mu, mu = 0; at the others
    mu += (sum of the 6 neighbours) / 6 (boundary entries hold 0)."""
    out = mu.copy()
    s = sum(_nb(mu, d) for d in _SH)
    on = par == color
    _in(muf)[on] += h2 / 6.0 * _in(mu)[on]
    _in(out)[on] = 0.0
    _in(out)[~on] = _in(mu)[~on] + s[~on] / 6.0
    return out, muf


def _adj_sweep(mu, muf, h2, par):
    """transpose of one forward sweep (colour 0, then colour 1)"""
    mu, muf = _adj_color(mu, muf, h2, 1, par)
    return _adj_color(mu, muf, h2, 0, par)


def _full_weighting(X, SC):
    """(1/64)(8,4,2,1) full weighting onto the coarse interior (coarse boundary 0)."""
    out = np.zeros((SC, SC, SC))
    n = SC - 1
    acc = np.zeros((n - 1, n - 1, n - 1))
    for a in (-1, 0, 1):
        for b in (-1, 0, 1):
            for c in (-1, 0, 1):
                w = (2.0 if a == 0 else 1.0) * (2.0 if b == 0 else 1.0) * (2.0 if c == 0 else 1.0)
                acc += w * X[2 + a:2 * n - 1 + a:2, 2 + b:2 * n - 1 + b:2, 2 + c:2 * n - 1 + c:2]
    out[1:-1, 1:-1, 1:-1] = acc / 64.0
    return out


def _trilinear(Ec, S):
    """trilinear interpolation of a coarse field onto the fine interior (fine boundary 0)."""
    out = np.zeros((S, S, S))
    i = np.arange(1, S - 1)
    lo, hi = i >> 1, (i >> 1) + (i & 1)
    V = 0.125 * sum(Ec[np.ix_(x, y, z)] for x in (lo, hi) for y in (lo, hi) for z in (lo, hi))
    out[1:-1, 1:-1, 1:-1] = V
    return out


def adj_vcycle(mu, S, h, levels, pre, post, coarse_sweeps):
    """Transpose of nm_vcycle_rec (oracle/rq_oracle.c): mu = dE/dP after the cycle -> (dE/dP
    before it, dE/df)."""
    h2 = h * h
    par = _colors(S)
    muf = np.zeros_like(mu)
    if levels <= 1:
        for _ in range(coarse_sweeps):
            mu, muf = _adj_sweep(mu, muf, h2, par)
        return mu, muf
    for _ in range(post):
        mu, muf = _adj_sweep(mu, muf, h2, par)
    SC = (S - 1) // 2 + 1
    muc = 8.0 * _full_weighting(mu, SC)                    # prolongation^T
    _, mufc = adj_vcycle(muc, SC, 2 * h, levels - 1, pre, post, coarse_sweeps)  # the coarse cycle starts at 0
    mur = _trilinear(mufc, S) / 8.0                         # full weighting^T
    muf = muf + mur                                         # residual^T
    lap = sum(_nb(mur, d) for d in _SH) - 6.0 * _in(mur)
    mu = mu.copy()
    _in(mu)[...] += lap / h2
    for _ in range(pre):
        mu, muf = _adj_sweep(mu, muf, h2, par)
    return mu, muf


def _adj_norm(psi, lam, c, L, Z, h3):
    """normalise^T at the normalised state psi with the forward per-domain scales c"""
    n = len(Z)
    Lc = np.clip(L, 0, n - 1)
    dots = np.bincount(Lc.reshape(-1), weights=(psi * lam).reshape(-1), minlength=n)
    beta = np.where(Z > 0, c * h3 * dots / np.where(Z > 0, Z, 1.0), 0.0)
    return c[Lc] * lam - beta[Lc] * psi


def _scales(drv):
    _, pd = drv.domain_sums()
    N, Z = pd[:, 0], drv.Zdom
    return np.where((Z > 0) & (N > 1e-300), np.sqrt(Z / np.where(N > 0, N, 1.0)), 1.0)


def gradient(drv, n_steps):
    """n_steps of drv with recording, then the reverse sweep.  Returns (E, F (n x 3), dE/dK (S^3))."""
    S, h, n = drv.S, drv.h, drv.n
    h3 = h ** 3
    shp = (S, S, S)
    L = drv.label.reshape(shp)
    Z = drv.Zdom
    recs = []
    for _ in range(n_steps):
        s = drv.steps_done + 1
        assert not (s % drv.li == 0 and (drv.label_until <= 0 or s <= drv.label_until)), "labels must be frozen"
        vc = s % drv.pi_ == 0
        norm = (s + 1) % drv.ni == 0 or (s + 1) % drv.pi_ == 0
        if vc:
            drv.vcycle()
        # the state the step starts from (normalised when the step before normalised)
        rec = {"psi": drv.U.copy(), "P": drv.P.copy(), "vc": vc, "norm": norm}
        drv.steps_done = s
        orc.O().nm_update(drv.U, drv.U2, drv.K, drv.P, drv.label, S, drv.half_dv, drv.dt)
        drv.U, drv.U2 = drv.U2, drv.U
        if norm:
            rec["c"] = _scales(drv)
            drv.normalize()
        else:
            drv.age += 1
        recs.append(rec)
    c_final = _scales(drv) if drv.age else None
    E = drv.energy()["E"]  # normalises when updates ran since the last normalisation
    psi = drv.U.reshape(shp)
    K, P = drv.K.reshape(shp), drv.P.reshape(shp)
    _, pd = drv.domain_sums()
    N = pd[:, 0]
    w = np.where((Z > 0) & (N > 0), Z / np.where(N > 0, N, 1.0), 1.0)
    Q = pd[:, 1] + pd[:, 2] + 2.0 * pd[:, 3]  # the readout's per-domain part, w Q (NewMethodDriver.energy)
    qn = np.where(N > 0, Q / np.where(N > 0, N, 1.0), 0.0)
    Lc = np.clip(L, 0, n - 1)
    lam = np.zeros(shp)
    muP = np.zeros(shp)
    gK = np.zeros(shp)
    wl, ql, u = _in(w[Lc]), _in(qn[Lc]), _in(psi)
    AP = (6.0 * _in(P) - sum(_nb(P, d) for d in _SH)) / (h * h)
    _in(lam)[...] = wl * (-h * _same_label_lap(psi, L) + 2.0 * h3 * u * (2.0 * _in(P) - _in(K) - ql))
    _in(muP)[...] = 2.0 * wl * h3 * u * u - h3 / math.pi * AP
    _in(gK)[...] = -wl * h3 * u * u
    if c_final is not None and recs:
        lam = _adj_norm(psi, lam, c_final, L, Z, h3)
    for r in range(len(recs) - 1, -1, -1):
        R = recs[r]
        pp = R["psi"].reshape(shp)
        if R["norm"]:
            ps = recs[r + 1]["psi"].reshape(shp) if r + 1 < len(recs) else psi
            lam = _adj_norm(ps, lam, R["c"], L, Z, h3)
        Ps = R["P"].reshape(shp)
        lt = lam
        lam = np.zeros(shp)
        _in(lam)[...] = _in(lt) + drv.half_dv * _same_label_lap(lt, L) + drv.dt * (_in(K) - 2.0 * _in(Ps)) * _in(lt)
        _in(gK)[...] += drv.dt * _in(pp) * _in(lt)
        _in(muP)[...] += -2.0 * drv.dt * _in(pp) * _in(lt)
        if R["vc"]:
            muP, muf = adj_vcycle(muP, S, h, drv.levels, drv.pre, drv.post, drv.cs)
            _in(lam)[...] += 4.0 * math.pi * _in(pp) * _in(muf)
    # F_a = sum_i gK_i dK_a/dr (x_i - R_a) / r
    from scipy.special import erf
    xyz, Zn = drv.nuclei()
    xyz = xyz.reshape(-1, 3)
    inv = 1.0 / (math.sqrt(2.0) * drv.sigma)
    gs = math.sqrt(2.0 / math.pi) / drv.sigma
    idx = np.arange(1, S - 1) * h
    X, Y, Zg = np.meshgrid(idx, idx, idx, indexing="ij")
    gi = _in(gK)
    F = np.zeros((n, 3))
    for a in range(n):
        if Zn[a] <= 0:
            continue
        dx, dy, dz = X - xyz[a, 0], Y - xyz[a, 1], Zg - xyz[a, 2]
        r2 = dx * dx + dy * dy + dz * dz
        ok = r2 > 1e-24
        rr = np.where(ok, np.sqrt(r2), 1.0)
        dKdr = Zn[a] * (gs * np.exp(-r2 * inv * inv) / rr - erf(rr * inv) / (rr * rr))
        wgt = np.where(ok, gi * dKdr / rr, 0.0)
        F[a] = [(wgt * dx).sum(), (wgt * dy).sum(), (wgt * dz).sum()]
    return E, F, gK.reshape(-1)
