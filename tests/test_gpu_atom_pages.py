"""What the atom.js H page converges to (atom_H.html: Z = 1, one shell, NN = 100, screen 10 bohr).

The page's model for one electron is ITP on -1/2 div(W grad) - K W + 2P W, with K = Z / sqrt(r^2 +
0.12 h^2) stored as f32 (atom.js:47-51), W = 1 inside the shell's ball r < 5 bohr (atom.js:60-80)
and P the Hartree potential of the OTHER shells: with one shell its right-hand side is zero, so
P's fixed point is 0.  The page starts P at 0.5 / r (atom.js:90, meant for the other shell of a
two-shell atom), which cancels the nuclear attraction at first and decays only through the
V-cycles -- the slow climb seen on the page (-0.406 Ha after 6000 steps).  With that remnant
removed (P = 0 uploaded) the energy settles within 0.01 Ha of the page's stated
-0.500: the rest is the grid (the unweighted discrete operator's lowest eigenvalue on this grid,
computed here independently with scipy, is -0.4968 Ha) and the shell's ball.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def discrete_ground_state(NN, screen, Z):
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    h = screen / NN
    n = NN - 1
    x = (np.arange(1, NN) - NN // 2) * h
    X, Y, Zc = np.meshgrid(x, x, x, indexing="ij")
    r = np.sqrt(X ** 2 + Y ** 2 + Zc ** 2 + 0.12 * h * h)
    K = (Z / r).astype(np.float32).astype(np.float64).ravel()
    e = np.ones(n)
    L1 = sp.diags([e[:-1], -2 * e, e[:-1]], [-1, 0, 1]) / (h * h)
    I1 = sp.identity(n)
    lap = sp.kron(sp.kron(L1, I1), I1) + sp.kron(sp.kron(I1, L1), I1) + sp.kron(sp.kron(I1, I1), L1)
    H = (-0.5 * lap - sp.diags(K)).tocsr()
    vals = sla.eigsh(H, k=1, which="SA", v0=np.exp(-r).ravel(), tol=1e-10, maxiter=20000)[0]
    return float(vals[0])


def test_h_page_without_the_hartree_remnant_reaches_the_stated_energy():
    from realmolecule_b200.shells import AtomShells
    s = AtomShells(NN=100, screen=10.0, Z_kernel=1.0, shells=[{"ne": 1, "Rmax": 5.0, "Zeff": 1}])
    f = s.fields(0)
    s.set_fields(0, U=f["U"], W=f["W"], P=np.zeros_like(f["P"]))
    E = [s.step(1000)["E"] for _ in range(3)]
    res = s.step(1)
    assert abs(res["E_ee"]) < 1e-9
    assert abs(E[2] - E[1]) < 2e-3 and abs(E[2] + 0.5) < 1e-2, E
    lam = discrete_ground_state(100, 10.0, 1.0)
    assert abs(lam - (-0.4968)) < 1e-3, lam
