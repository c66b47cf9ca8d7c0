"""A second, pure-Python restatement of atom.js's physicsStep (atom.js:213-333) with the
simultaneous Poisson update, written from the JavaScript text independently of oracle/rq_oracle.c:
JavaScript numbers (double) over Float32Array storage (every store rounds to f32; c[] is a
Float32Array too), the in-place lexicographic sweep, the front speed c[m] with its reassignment
inside the n loop, the domain-dominance energy sums and the per-shell normalisation.  Compared
with the C restatement after one step on a small grid (CPU): fields bit for bit, energies to
1e-12."""
import math

import numpy as np
import pytest

import oracle as orc

f32 = np.float32


def physics_step(U, W, P, K, fixed, NN, h, d):
    """U, W, P: lists of per-shell float32 arrays (modified in place)."""
    n = len(U)
    S = NN + 1
    S2 = S * S
    h2, h3 = h * h, h * h * h
    dt = d * h2
    c = np.zeros(n, np.float32)
    ET = Eee = EeK = 0.0
    for i in range(1, NN):
        for j in range(1, NN):
            for k in range(1, NN):
                idx = i * S2 + j * S + k
                for m in range(n):
                    c[m] = 0
                    for q in range(n):
                        if q != m:
                            c[m] = float(c[m]) - float(U[q][idx])
                        c[m] = 0.5 * (float(c[m]) + float(U[m][idx]))
                ip, im, jp, jm, kp, km = idx + S2, idx - S2, idx + S, idx - S, idx + 1, idx - 1
                for m in range(n):
                    u, w, pm = U[m], W[m], P[m]
                    if not fixed[m]:
                        lapW = (float(w[ip]) + float(w[im]) + float(w[jp]) + float(w[jm]) + float(w[kp])
                                + float(w[km]) - 6 * float(w[idx])) / h2
                        gwx = (float(w[ip]) - float(w[im])) / h
                        gwy = (float(w[jp]) - float(w[jm])) / h
                        gwz = (float(w[kp]) - float(w[km])) / h
                        gradW = math.sqrt(gwx * gwx + gwy * gwy + gwz * gwz)
                        w[idx] = float(w[idx]) + (2 * dt * abs(float(c[m])) * lapW + 9 * dt * float(c[m]) * gradW)
                    U0, W0 = float(u[idx]), float(w[idx])
                    wlap = (0.5 * d * ((float(u[ip]) - U0) * (float(w[ip]) + W0) * 0.5
                                       - (U0 - float(u[im])) * (W0 + float(w[im])) * 0.5)
                            + 0.5 * d * ((float(u[jp]) - U0) * (float(w[jp]) + W0) * 0.5
                                         - (U0 - float(u[jm])) * (W0 + float(w[jm])) * 0.5)
                            + 0.5 * d * ((float(u[kp]) - U0) * (float(w[kp]) + W0) * 0.5
                                         - (U0 - float(u[km])) * (W0 + float(w[km])) * 0.5))
                    u[idx] = U0 + (wlap + dt * (float(K[idx]) - 2 * float(pm[idx])) * U0 * W0)
                    Wm = float(w[idx])
                    dominated = all(not (q != m and float(W[q][idx]) >= Wm) for q in range(n))
                    if dominated and Wm > 0.01:
                        dom = []
                        for nb in (ip, jp, kp):
                            dom.append(all(not (q != m and float(W[q][nb]) >= float(w[nb])) for q in range(n)))
                        gx = float(u[ip]) - float(u[idx]) if dom[0] else 0
                        gy = float(u[jp]) - float(u[idx]) if dom[1] else 0
                        gz = float(u[kp]) - float(u[idx]) if dom[2] else 0
                        ET += 0.5 * (gx * gx + gy * gy + gz * gz) * h
                        Eee += float(pm[idx]) * float(u[idx]) * float(u[idx]) * h3
                        EeK += -float(K[idx]) * float(u[idx]) * float(u[idx]) * h3
                    rho_o = 0.0
                    for q in range(n):
                        if q != m:
                            rho_o += float(U[q][idx]) * float(U[q][idx]) * float(W[q][idx])
                    lapP = (float(pm[ip]) + float(pm[im]) + float(pm[jp]) + float(pm[jm]) + float(pm[kp])
                            + float(pm[km]) - 6 * float(pm[idx])) / h2
                    pm[idx] = float(pm[idx]) + (dt * lapP + 2 * math.pi * dt * rho_o)
    for m in range(n):
        n2 = 0.0
        for i in range(1, NN):
            for j in range(1, NN):
                for k in range(1, NN):
                    n2 += float(U[m][i * S2 + j * S + k]) ** 2 * h3
        sc = 1 / math.sqrt(n2)
        for i in range(1, NN):
            for j in range(1, NN):
                for k in range(1, NN):
                    U[m][i * S2 + j * S + k] = float(U[m][i * S2 + j * S + k]) * sc
    return ET + EeK + Eee, ET, EeK, Eee


@pytest.mark.parametrize("shells", [
    [{"ne": 1, "Rmax": 1.0, "Zeff": 2}, {"ne": 1, "Rmax": 2.0, "Zeff": 1}],
    [{"ne": 1, "Rmax": 1.5, "Zeff": 2, "split": "halfspace", "halfIndex": 0, "fixedW": True},
     {"ne": 1, "Rmax": 1.5, "Zeff": 2, "split": "halfspace", "halfIndex": 1, "fixedW": True}],
], ids=["radial_fronts", "halfspace_fixed"])
def test_physics_step_matches_a_python_restatement(shells):
    NN, scr, Z, d = 12, 3.0, 2, 0.1
    ref = orc.AtomShellsDriver(NN, scr, Z, shells, d=d, poisson="simultaneous")
    ref.initialize()
    S3 = ref.S3
    n = len(shells)
    U = [ref.U[m * S3:(m + 1) * S3].copy() for m in range(n)]
    W = [ref.W[m * S3:(m + 1) * S3].copy() for m in range(n)]
    P = [ref.P[m * S3:(m + 1) * S3].copy() for m in range(n)]
    K = ref.K.copy()
    want = physics_step(U, W, P, K, [bool(s.get("fixedW")) for s in shells], NN, scr / NN, d)
    E4, _ = ref.step()
    for m in range(n):
        sl = slice(m * S3, (m + 1) * S3)
        assert np.array_equal(ref.U[sl].view(np.uint32), U[m].view(np.uint32)), ("U", m)
        assert np.array_equal(ref.W[sl].view(np.uint32), W[m].view(np.uint32)), ("W", m)
        assert np.array_equal(ref.P[sl].view(np.uint32), P[m].view(np.uint32)), ("P", m)
    for a, b in zip(E4, want):
        assert abs(a - b) <= 1e-12 * max(1.0, abs(b)), (E4, want)
