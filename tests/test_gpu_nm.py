"""New flavour (Gaussian nuclei, red-black multigrid, FP64 domain sums) on the GPU against the
FP64 oracle of the same method (oracle.NewMethodDriver), plus mixed-vs-FP64 energy agreement and
forces against central finite differences of the converged energy.

Bars: FP64 path -- labels and the multigrid V-cycle bit-exact (same operations in the same
order; the per-domain sums and erf/exp are the only order/ulp differences), psi and energies
within 1e-11 relative.  Mixed path -- converged energy within 1e-6 relative of the FP64 path.
Forces -- within 1e-4 Ha/bohr of central differences (delta = 1e-3 bohr) of the converged
FP64 energy with labels frozen.
"""
import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu


def water_rows(NN=32, h=0.5):
    from realmolecule_b200 import configs as C
    g = C.h2o64()
    g.NN, g.h = NN, h
    return NN, g.screen, C.to_domain_atoms(g)


def h2_rows(NN=32, h=0.3, R=1.4):
    N2 = NN / 2
    d = R / 2 / h
    return NN, NN * h, [
        {"i": N2 - d, "j": N2, "k": N2, "Z": 0.0, "Z_nuc": 1.0},
        {"i": N2 + d, "j": N2 + 0.01, "k": N2, "Z": 0.0, "Z_nuc": 1.0},
        {"i": N2 - d + 0.05, "j": N2, "k": N2, "Z": 1.0, "Z_nuc": 0.0},
        {"i": N2 + d - 0.05, "j": N2, "k": N2, "Z": 1.0, "Z_nuc": 0.0}]


def ctx_for(NN, screen, rows, precision="fp64", **kw):
    from realmolecule_b200 import Context
    return Context(NN, screen, rows, flavor="new", precision=precision, **kw)


def test_initial_state_fp64():
    from realmolecule_b200 import _lib as L
    NN, scr, rows = water_rows()
    ref = orc.NewMethodDriver(NN, scr, rows)
    ref.initialize()
    ctx = ctx_for(NN, scr, rows)
    ctx.initialize()
    st = ctx.download(psi=True, label=True, P=True)
    assert np.array_equal(st["label"], ref.label)
    np.testing.assert_allclose(ctx.download_K(), ref.K, rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(st["psi"], ref.U, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(st["P"], ref.P, rtol=1e-11, atol=1e-14)
    e = ctx.energy()
    o = ref.energy()
    for k, v in ((L.E_T, o["T"]), (L.E_EK, o["EK"]), (L.E_EE, o["EE"]), (L.E_KK, o["KK"])):
        assert abs(e[k] - v) <= 1e-11 * max(1, abs(v)), (k, e[k], v)


def test_vcycle_bit_exact_fp64():
    NN, scr, rows = water_rows()
    ref = orc.NewMethodDriver(NN, scr, rows, poisson_interval=1)
    ref.initialize()
    ctx = ctx_for(NN, scr, rows, poisson_interval=1, label_interval=1000)
    ctx.initialize()
    ctx.upload(psi=ref.U, label=ref.label, P=np.zeros_like(ref.P))
    P0 = np.zeros_like(ref.P)
    orc.O().nm_vcycle(P0, ref.U, ref.S, ref.h, ref.levels, ref.pre, ref.post, ref.cs)
    ctx.step(1)  # V-cycle on the uploaded psi, then the update
    P = ctx.download(psi=False, label=False, P=True)["P"]
    assert np.array_equal(P.view(np.uint64), P0.view(np.uint64))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_steps_against_oracle(precision):
    NN, scr, rows = water_rows()
    ref = orc.NewMethodDriver(NN, scr, rows, label_interval=10)
    ref.initialize()
    ctx = ctx_for(NN, scr, rows, precision=precision, label_interval=10)
    ctx.initialize()
    for _ in range(60):
        ref.step()
    ctx.step(60)
    st = ctx.download(psi=True, label=True)
    mism = (st["label"] != ref.label).sum()
    assert mism <= (0 if precision == "fp64" else 50), mism
    tol = 1e-10 if precision == "fp64" else 2e-4
    assert np.max(np.abs(st["psi"] - ref.U)) <= tol * np.abs(ref.U).max()


def converge(ctx, tol=1e-10, max_steps=20000):
    steps, E = ctx.solve(tol, max_steps, 100)
    assert steps < max_steps, "did not converge"
    return E


def test_mixed_matches_fp64_converged_energy():
    NN, scr, rows = water_rows()
    E = {}
    for p in ("fp64", "mixed"):
        ctx = ctx_for(NN, scr, rows, precision=p, label_until=400)
        ctx.initialize()
        ctx.step(400)
        E[p] = converge(ctx, tol=1e-9 if p == "fp64" else 1e-7)
    assert abs(E["mixed"] - E["fp64"]) <= 1e-6 * abs(E["fp64"]), E


def test_promoted_mixed_solve_reaches_the_fp64_fixed_point():
    """fp32 fields stall a few 1e-8 |E| above the FP64 fixed point; continuing in FP64 from the
    mixed state (rq_promote) reaches it."""
    NN, scr, rows = water_rows()
    ref = ctx_for(NN, scr, rows, precision="fp64", label_until=1)
    ref.initialize()
    ref.step(6000)
    E64 = float(ref.energy()[0])
    ref.close()
    ctx = ctx_for(NN, scr, rows, precision="mixed", label_until=1)
    ctx.initialize()
    ctx.step(2000)
    psi32 = ctx.download(psi=True)["psi"]
    ctx.promote()
    assert ctx.fp64
    psi64 = ctx.download(psi=True)["psi"]
    assert psi64.dtype == np.float64 and np.array_equal(psi64.astype(np.float32), psi32)
    ctx.step(4000)
    E = float(ctx.energy()[0])
    ctx.promote()  # a no-op on an FP64 context
    ctx.close()
    assert abs(E - E64) <= 1e-9 * abs(E64), (E, E64)


def test_adjoint_force_matches_finite_differences():
    from realmolecule_b200 import _lib as L
    NN, scr, rows = h2_rows()
    h = scr / NN
    ctx = ctx_for(NN, scr, rows, label_until=1)
    ctx.initialize()
    converge(ctx, tol=1e-12)
    Fe = ctx.forces(L.FORCE_ADJOINT)
    _, Fn = ctx.nuclear_terms()
    F = Fe + Fn
    delta = 1e-3
    for a, axis in ((0, 0), (1, 1), (1, 0)):
        Es = []
        for sgn in (+1, -1):
            r2 = [dict(r) for r in rows]
            r2[a]["ijk"[axis]] += sgn * delta / h
            ctx.set_atoms(r2)
            Es.append(converge(ctx, tol=1e-13))
        ctx.set_atoms(rows)
        fd = -(Es[0] - Es[1]) / (2 * delta)
        assert abs(fd - F[a, axis]) < 1e-4, (a, axis, fd, F[a, axis])
    # and the GPU force equals the oracle's on the same psi
    st = ctx.download(psi=True, label=False)
    xyz = np.array([[r["i"] * h, r["j"] * h, r["k"] * h] for r in rows]).reshape(-1)
    Z = np.array([r["Z_nuc"] for r in rows])
    Fo = np.zeros(len(rows) * 3)
    orc.O().nm_force(st["psi"], xyz, Z, len(rows), NN + 1, h, h, Fo)
    np.testing.assert_allclose(ctx.forces(L.FORCE_ADJOINT).reshape(-1), Fo, rtol=1e-9, atol=1e-12)
