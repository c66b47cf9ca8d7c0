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
