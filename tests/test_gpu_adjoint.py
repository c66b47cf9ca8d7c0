"""The new flavour's adjoint (rq_set_adjoint_window / rq_adjoint) on the GPU: against the FP64
restatement of the same reverse sweep (oracle/nm_adjoint.py), and against central finite
differences of the energy it differentiates -- the energy read out after N warm-started
imaginary-time steps from a fixed, NOT converged state (labels frozen), as a function of the
nuclear positions and of an external potential.

Every finite difference restarts from the same uploaded state and runs the same N steps in the
same schedule phase, so E(R) is one deterministic function; in FP64 its central difference
(delta = 1e-3 bohr) carries ~1e-8 Ha/bohr of truncation and rounding error.  Bar (the force
tolerance of the benchmark configurations): 1e-4 Ha/bohr.  With an empty window the adjoint is
the Hellmann-Feynman gather (the form of the reference's force routines, cloud/solver.py:282-315
and molecule.js:1271-1330), which the convergence test checks at a converged state.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_STEPS = 48  # a multiple of the V-cycle period (4): every restart runs the same schedule phase
DELTA = 1e-3


def _prepared(NN, screen, rows, precision="fp64", settle=400, extra=200):
    """A context whose labels have settled and are frozen, a few hundred steps short of convergence."""
    from realmolecule_b200 import Context
    ctx = Context(NN, screen, rows, flavor="new", precision=precision, label_until=settle)
    ctx.initialize()
    ctx.step(settle + extra)
    st = ctx.download(psi=True, label=False, P=True)
    return ctx, st


def _energy_after(ctx, st, rows, steps=N_STEPS, v=None):
    from realmolecule_b200 import _lib as L
    ctx.upload(psi=st["psi"], P=st["P"])
    ctx.set_atoms(rows)
    if v is not None:
        ctx.set_external_potential(v)
    ctx.step(steps)
    return float(ctx.energy()[L.E_TOTAL])


def _water_pair_rows(NN=40, h=0.3):
    """Two waters (6 nuclei, 20 domains): a small cluster of the kind the dynamics workloads step."""
    from realmolecule_b200 import configs as C
    g = C.h2o64()
    rot = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    shift = np.array([2.9, 0.4, 0.3])  # bohr: the second water turned by 90 degrees and moved
    xyz = np.concatenate([g.xyz, g.xyz @ rot.T + shift])
    seeds = np.concatenate([g.seeds, g.seeds @ rot.T + shift])
    centre = xyz.mean(0)
    gg = C.Geometry("water2", g.elements * 2, xyz - centre, NN, h)
    gg.seeds = seeds - centre
    return NN, NN * h, C.to_domain_atoms(gg)


def _fd_forces(ctx, st, rows, coords, h):
    F = {}
    for (a, ax) in coords:
        E = []
        for sgn in (+1, -1):
            r2 = [dict(r) for r in rows]
            r2[a]["ijk"[ax]] += sgn * DELTA / h
            E.append(_energy_after(ctx, st, r2))
        F[(a, ax)] = -(E[0] - E[1]) / (2 * DELTA)
    return F


def test_gpu_adjoint_matches_the_oracle_adjoint():
    """The CUDA reverse sweep against the FP64 restatement from one uploaded state: energy 1e-12
    relative, forces and dE/dK within 1e-9 of their largest value."""
    import oracle as orc
    import nm_adjoint as adj
    from realmolecule_b200 import Context, _lib as L
    NN, h = 16, 0.45
    N2, d = NN / 2, 1.4 / 2 / h
    rows = [{"i": N2 - d, "j": N2, "k": N2 + 0.2, "Z": 0.0, "Z_nuc": 1.0},
            {"i": N2 + d, "j": N2 + 0.3, "k": N2, "Z": 0.0, "Z_nuc": 1.0},
            {"i": N2 - d + 0.05, "j": N2, "k": N2, "Z": 1.0, "Z_nuc": 0.0},
            {"i": N2 + d - 0.05, "j": N2, "k": N2, "Z": 1.0, "Z_nuc": 0.0}]
    drv = orc.NewMethodDriver(NN, NN * h, rows, label_until=40)
    drv.initialize()
    for _ in range(60):
        drv.step()
    drv.ready()
    ctx = Context(NN, NN * h, rows, flavor="new", precision="fp64", label_until=40)
    ctx.initialize()
    ctx.step(60)  # the same schedule phase, labels frozen from here on
    ctx.set_adjoint_window(N_STEPS)
    ctx.upload(psi=drv.U, label=drv.label, P=drv.P)
    ctx.set_atoms(rows)
    ctx.step(16)
    E = float(ctx.energy()[L.E_TOTAL])
    F, g = ctx.adjoint(forces=True, potential=True)
    Eo, Fo, go = adj.gradient(drv, 16)
    assert abs(E - Eo) <= 1e-12 * abs(Eo)
    assert np.max(np.abs(F - Fo)) <= 1e-9 * np.max(np.abs(Fo))
    assert np.max(np.abs(g - go)) <= 1e-9 * np.max(np.abs(go))
    ctx.close()


def test_adjoint_matches_finite_differences_after_warm_started_steps():
    NN, screen, rows = _water_pair_rows()
    h = screen / NN
    ctx, st = _prepared(NN, screen, rows)
    ctx.set_adjoint_window(N_STEPS)
    _energy_after(ctx, st, rows)
    Fe, _ = ctx.adjoint()
    _, Fn = ctx.nuclear_terms()
    F = Fe + Fn
    nuclei = [q for q, r in enumerate(rows) if r["Z_nuc"] > 0]
    coords = [(a, ax) for a in nuclei for ax in range(3)]
    fd = _fd_forces(ctx, st, rows, coords, h)
    err = max(abs(fd[c] - F[c]) for c in coords)
    assert err < 1e-4, err
    # the finite differences see the non-converged iteration: the Hellmann-Feynman force alone misses it
    ctx.set_adjoint_window(0)
    _energy_after(ctx, st, rows)
    Fhf = ctx.forces(0) + Fn
    assert max(abs(fd[c] - Fhf[c]) for c in coords) > 10 * err
    ctx.close()


def test_adjoint_potential_gradient_matches_finite_differences():
    NN, screen, rows = _water_pair_rows(NN=32, h=0.35)
    ctx, st = _prepared(NN, screen, rows, settle=200, extra=100)
    S = NN + 1
    x = np.arange(S) * (screen / NN) - screen / 2
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    w = (0.05 * np.exp(-((X - 0.7) ** 2 + (Y + 0.3) ** 2 + Z ** 2) / 4.0)).reshape(-1)
    ctx.set_adjoint_window(N_STEPS)
    _energy_after(ctx, st, rows, v=np.zeros(S ** 3))
    _, g = ctx.adjoint(forces=False, potential=True)
    eps = 1e-3
    Ep = _energy_after(ctx, st, rows, v=eps * w)
    Em = _energy_after(ctx, st, rows, v=-eps * w)
    fd = (Ep - Em) / (2 * eps)
    ad = float(np.dot(g, w))
    assert abs(fd - ad) <= 1e-6 * max(1.0, abs(fd)), (fd, ad)
    ctx.close()


def test_empty_window_is_the_hellmann_feynman_gather():
    from realmolecule_b200 import _lib as L
    NN, screen, rows = _water_pair_rows(NN=32, h=0.35)
    ctx, _ = _prepared(NN, screen, rows, settle=200, extra=100)
    ctx.set_adjoint_window(8)
    ctx.set_atoms(rows)  # resets the window: no recorded step
    Fa, _ = ctx.adjoint()
    Fh = ctx.forces(L.FORCE_HF)
    np.testing.assert_allclose(Fa, Fh, rtol=1e-9, atol=1e-12)
    ctx.close()


def test_adjoint_reaches_hellmann_feynman_at_convergence():
    """From a converged state the gradient of the energy after N more steps is the Hellmann-Feynman
    force (the form of the reference's force routine): the readout is stationary in psi and, in its
    P-stationary Hartree form, in P.  Bar: 1e-6 Ha/bohr for windows of 48 and 2000 steps."""
    from realmolecule_b200 import _lib as L
    NN, screen, rows = _water_pair_rows(NN=32, h=0.35)
    ctx, _ = _prepared(NN, screen, rows, settle=200, extra=100)
    ctx.solve(1e-13, 60000, 200)
    Fh = ctx.forces(L.FORCE_HF)
    gaps = []
    for n in (N_STEPS, 2000):
        ctx.set_adjoint_window(n)
        ctx.set_atoms(rows)
        ctx.step(n)
        Fa, _ = ctx.adjoint()
        gaps.append(np.max(np.abs(Fa - Fh)))
    assert max(gaps) < 1e-6, gaps
    ctx.close()


def test_glycine_all_30_coordinates_against_finite_differences():
    """Glycine (10 nuclei, 40 domains) on 128^3 at h = 0.2 bohr, FP64: the adjoint force on all 30
    nuclear coordinates against central differences (delta = 1e-3 bohr) of the energy after
    N_STEPS warm-started steps."""
    from realmolecule_b200 import configs as C
    g = C.glycine128()
    rows = C.to_domain_atoms(g)
    ctx, st = _prepared(g.NN, g.screen, rows, settle=400, extra=400)
    ctx.set_adjoint_window(N_STEPS)
    _energy_after(ctx, st, rows)
    Fe, _ = ctx.adjoint()
    _, Fn = ctx.nuclear_terms()
    F = Fe + Fn
    coords = [(a, ax) for a in range(len(g.elements)) for ax in range(3)]
    fd = _fd_forces(ctx, st, rows, coords, g.h)
    errs = np.array([abs(fd[c] - F[c]) for c in coords])
    assert errs.max() < 1e-4, errs.max()
    ctx.close()
