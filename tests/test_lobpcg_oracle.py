"""The oracle's restatement of molecule.js's LOBPCG frame (molecule.js:1455-1724, :3265-3740) on
CPU: the Ritz solvers against a generalized symmetric eigensolver, the inner products against
FP64 dot products, and whole frames on a small grid.  The GPU path is compared with these
functions bit for bit in test_gpu_mj.py."""
import numpy as np
import pytest
import scipy.linalg as sl

import oracle as orc


def ip_vector(S, H):
    """The 12 sums in the shaders' order from 3x3 Gram (S) and Hamiltonian (H) matrices over
    (X, W, P): <X|X> <X|HX> <W|W> <W|HW> <X|W> <X|HW> <P|P> <P|HP> <X|P> <X|HP> <W|P> <W|HP>."""
    return np.array([S[0, 0], H[0, 0], S[1, 1], H[1, 1], S[0, 1], H[0, 1], S[2, 2], H[2, 2], S[0, 2], H[0, 2],
                     S[1, 2], H[1, 2]], np.float64)


@pytest.mark.parametrize("seed", range(5))
def test_ritz_solvers_give_the_lowest_generalized_eigenpair(seed):
    rng = np.random.default_rng(seed)
    for _ in range(40):
        B = rng.normal(size=(40, 3))
        S = B.T @ B / 40
        H = rng.normal(size=(3, 3))
        H = H + H.T
        ip = ip_vector(S, H)
        out = np.zeros(4)
        orc.O().lob_ritz3(ip, out)
        lam = sl.eigh(H, S, eigvals_only=True)[0]
        c = out[1:]
        assert abs(out[0] - lam) <= 1e-12 * max(1.0, abs(lam))
        assert abs(c @ S @ c - 1.0) <= 1e-12
        np.testing.assert_allclose(H @ c, lam * (S @ c), atol=1e-9 * max(1.0, abs(lam)))
        orc.O().lob_ritz2(ip, out)
        lam2 = sl.eigh(H[:2, :2], S[:2, :2], eigvals_only=True)[0]
        assert abs(out[0] - lam2) <= 1e-12 * max(1.0, abs(lam2)) and out[3] == 0.0


def test_ritz3_fallback_only_for_a_factor_that_is_not_finite():
    """molecule.js:3318-3322 falls back to the 2x2 problem when the Cholesky factor is not finite
    or a diagonal is below 1e-15.  The factor's diagonals are clamped to sqrt(1e-30), which is
    exactly 1e-15 in double, so a dependent P still takes the 3x3 path; an infinite <P|P> falls
    back."""
    rng = np.random.default_rng(7)
    B = rng.normal(size=(30, 3))
    S = B.T @ B / 30
    H = rng.normal(size=(3, 3))
    H = H + H.T
    a, b = np.zeros(4), np.zeros(4)
    ip = ip_vector(S, H)
    ip[6] = np.inf
    orc.O().lob_ritz3(ip, a)
    orc.O().lob_ritz2(ip, b)
    assert np.array_equal(a, b) and b[3] == 0.0
    Bd = np.column_stack([B[:, :2], B[:, 0]])  # P = X: S singular, the clamp keeps the 3x3 path
    Sd = Bd.T @ Bd / 30
    ipd = ip_vector(Sd, H)
    orc.O().lob_ritz3(ipd, a)
    orc.O().lob_ritz2(ipd, b)
    assert not np.array_equal(a, b)


def test_inner_products_are_the_domain_dot_products():
    NN, S = 24, 25
    rng = np.random.default_rng(3)
    fields = [rng.normal(size=S ** 3).astype(np.float32) for _ in range(6)]
    label = rng.integers(0, 3, S ** 3).astype(np.uint32)
    h3 = np.float32(0.125)
    out = np.zeros(12, np.float32)
    orc.O().lob_inner(*fields, label, 1, S, h3, out)
    X, HX, W, HW, P, HP = (f.reshape(S, S, S)[1:-1, 1:-1, 1:-1].astype(np.float64) for f in fields)
    sel = label.reshape(S, S, S)[1:-1, 1:-1, 1:-1] == 1
    pairs = [(X, X), (X, HX), (W, W), (W, HW), (X, W), (X, HW), (P, P), (P, HP), (X, P), (X, HP), (W, P), (W, HP)]
    ref = np.array([np.sum(a[sel] * b[sel]) * float(h3) for a, b in pairs])
    np.testing.assert_allclose(out, ref, rtol=2e-5, atol=2e-4)


def test_lobpcg_frames_on_a_small_grid():
    rows = [{"i": 12, "j": 12, "k": 12, "Z": 6, "Z_nuc": 6, "rc": 0.4},
            {"i": 15, "j": 9, "k": 12, "Z": 1, "Z_nuc": 1, "rc": 0.0},
            {"i": 9, "j": 9, "k": 12, "Z": 1, "Z_nuc": 1, "rc": 0.0}]
    d = orc.MoleculeJsDriver(24, 6.0, rows, steps_per_frame=3, lobpcg=True)
    d.initialize()
    U0 = d.U.copy()
    for _ in range(2):
        d.step()
    assert d.frame == 2 and d.steps_done == 2
    assert np.isfinite(d.U).all() and not np.array_equal(d.U, U0)
    assert np.abs(d.LP).max() > 0  # a search direction carried into the next frame
    assert np.isfinite(d.total_energy())


def _lobpcg_case(seed=4, S=10):
    rng = np.random.default_rng(seed)
    n = S ** 3
    f = lambda: rng.normal(size=n).astype(np.float32)  # noqa: E731
    label = rng.integers(0, 3, n).astype(np.uint32)
    rows = [{"i": 3, "j": 4, "k": 5, "Z": 1.0, "rc": 0.6}, {"i": 6, "j": 6, "k": 3, "Z": 1.0, "rc": 0.0},
            {"i": 5, "j": 2, "k": 6, "Z": 2.0, "rc": 0.45}]
    return S, label, rows, f


def test_apply_h_residual_update_match_a_python_restatement():
    """applyH, lobpcgResidual and lobpcgUpdate (molecule.js:1483-1525, :1652-1724) restated again in
    f32 Python steps from the shader text: bit-equal to the C restatement."""
    S, label, rows, f = _lobpcg_case()
    h, inv_h2 = np.float32(0.3), np.float32(1 / 0.09)
    atoms = orc.mj_atoms(rows)
    U, K, Pot = f(), np.abs(f()), f()
    HU = np.zeros_like(U)
    orc.O().lob_apply_h(U, HU, K, label, Pot, orc.C.addressof(atoms), S, h, inv_h2)
    f32 = np.float32

    def inside(i, j, k, l):
        a = rows[l]
        if a.get("rc", 0) <= 0:
            return False
        d = [f32(f32(f32(c) - f32(p)) * h) for c, p in zip((i, j, k), (a["i"], a["j"], a["k"]))]
        return f32(np.sqrt(f32(f32(f32(d[0] * d[0]) + f32(d[1] * d[1])) + f32(d[2] * d[2])))) < f32(a["rc"])

    L3, U3 = label.reshape(S, S, S), U.reshape(S, S, S)
    for i in range(1, S - 1):
        for j in range(1, S - 1):
            for k in range(1, S - 1):
                idx = (i * S + j) * S + k
                my = int(L3[i, j, k])
                if inside(i, j, k, my):
                    want = f32(0)
                else:
                    uc = U3[i, j, k]
                    acc = None
                    for (a, b, c) in ((i + 1, j, k), (i - 1, j, k), (i, j + 1, k), (i, j - 1, k), (i, j, k + 1),
                                      (i, j, k - 1)):
                        ln = int(L3[a, b, c])
                        v = U3[a, b, c] if ln == my and not inside(a, b, c, ln) else uc
                        acc = v if acc is None else f32(acc + v)
                    lap = f32(acc - f32(f32(6) * uc))
                    want = f32(f32(f32(f32(-0.5) * lap) * inv_h2) + f32(f32(-K[idx] + f32(f32(2) * Pot[idx])) * uc))
                assert HU[idx].view(np.uint32) == np.float32(want).view(np.uint32), (i, j, k)
    W = np.zeros_like(U)
    lam = np.float32(-0.37)
    orc.O().lob_residual(U, HU, W, label, K, Pot, lam, 1, S, inv_h2)
    X, Pv = U.copy(), f()
    X0, P0 = X.copy(), Pv.copy()
    c = [np.float32(v) for v in (0.9, -0.4, 0.25)]
    orc.O().lob_update(X, W, Pv, label, c[0], c[1], c[2], 1, S)
    for idx in range(S ** 3):
        i, j, k = idx // (S * S), (idx // S) % S, idx % S
        if not (0 < i < S - 1 and 0 < j < S - 1 and 0 < k < S - 1):
            continue
        if label[idx] != 1:
            assert W[idx] == 0 and X[idx] == X0[idx] and Pv[idx] == P0[idx]
            continue
        r = f32(HU[idx] - f32(lam * X0[idx]))
        diag = f32(f32(f32(f32(3) * inv_h2) + f32(abs(f32(-K[idx] + f32(f32(2) * Pot[idx]))))) + f32(0.1))
        assert W[idx].view(np.uint32) == f32(r / diag).view(np.uint32)
        x, w, p = X0[idx], W[idx], P0[idx]
        assert X[idx].view(np.uint32) == f32(f32(f32(c[0] * x) + f32(c[1] * w)) + f32(c[2] * p)).view(np.uint32)
        assert Pv[idx].view(np.uint32) == f32(f32(c[1] * w) + f32(c[2] * p)).view(np.uint32)


def test_inner_product_tree_matches_a_python_restatement():
    """lobpcgInner + lobpcgFinalize's workgroup trees (molecule.js:1535-1648) restated in Python:
    the 12 f32 sums are bit-equal to the C restatement (here 4 workgroups of 128)."""
    S, label, rows, f = _lobpcg_case(seed=9, S=10)
    F = [f() for _ in range(6)]
    h3 = np.float32(0.027)
    got = np.zeros(12, np.float32)
    orc.O().lob_inner(*F, label, 2, S, h3, got)
    NM = S - 2
    tot = NM ** 3
    nwg = min(256, -(-tot // 128))
    pairs = [(0, 0), (0, 1), (2, 2), (2, 3), (0, 2), (0, 3), (4, 4), (4, 5), (0, 4), (0, 5), (2, 4), (2, 5)]
    part = []
    for w in range(nwg):
        sn = [[np.float32(0)] * 12 for _ in range(128)]
        for lid in range(128):
            cell = w * 128 + lid
            while cell < tot:
                k, j, i = cell % NM + 1, (cell // NM) % NM + 1, cell // (NM * NM) + 1
                idx = (i * S + j) * S + k
                if label[idx] == 2:
                    for q, (a, b) in enumerate(pairs):
                        sn[lid][q] = np.float32(sn[lid][q] + np.float32(np.float32(F[a][idx] * F[b][idx]) * h3))
                cell += nwg * 128
        s = 64
        while s > 0:
            for lid in range(s):
                sn[lid] = [np.float32(x + y) for x, y in zip(sn[lid], sn[lid + s])]
            s //= 2
        part.append(sn[0])
    wg = [[np.float32(0)] * 12 for _ in range(128)]
    for lid in range(128):
        for w in range(lid, nwg, 128):
            wg[lid] = [np.float32(x + y) for x, y in zip(wg[lid], part[w])]
    s = 64
    while s > 0:
        for lid in range(s):
            wg[lid] = [np.float32(x + y) for x, y in zip(wg[lid], wg[lid + s])]
        s //= 2
    assert np.array_equal(np.array(wg[0], np.float32).view(np.uint32), got.view(np.uint32))
