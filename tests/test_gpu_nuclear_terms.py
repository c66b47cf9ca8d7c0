"""Nuclear terms of the new flavour at the geometry workloads' sizes, on the GPU against the FP64
oracle: the Gaussian-nucleus potential K = sum Z erf(r / (sqrt2 sigma)) / r and the
Hellmann-Feynman force gather -h^3 sum rho dK/dr (x - R) / r.

The 100-water geometry (300 nuclei) on a 96^3 grid takes the tiled sums (nuclei near each 32^3
tile direct, the rest through Chebyshev node values), the small cases the direct ones; both are
checked, and against each other.

Bars: K within 1e-12 relative of the oracle (FP64 path) and the fp32 K within one fp32 ulp of
the rounded oracle value (mixed path); forces within 1e-10 relative to the largest component,
for the FP64 fields and for the fp32 fields (the oracle then gathers over the same fp32 psi
widened to FP64, so the comparison isolates the gather's own arithmetic); adjoint forces and
dE/dv of the tiled and direct gathers within 1e-10 relative.
"""
import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu


def water100_rows(NN=96, h=0.4):
    from realmolecule_b200 import configs as C
    g = C.water100()
    g.NN, g.h = NN, h  # the 100-water box (38.4 bohr) on a coarser grid, so the oracle runs in seconds
    return NN, NN * h, C.to_domain_atoms(g)


def ctx_for(NN, screen, rows, precision, **kw):
    from realmolecule_b200 import Context
    return Context(NN, screen, rows, flavor="new", precision=precision, **kw)


AUTO, DIRECT, TILED = 0, 1, 2


@pytest.fixture(scope="module")
def water100_oracle():
    NN, scr, rows = water100_rows()
    ref = orc.NewMethodDriver(NN, scr, rows)
    ref.initialize()
    return NN, scr, rows, ref


@pytest.mark.parametrize("mode", [AUTO, DIRECT])
def test_potential_fp64_matches_oracle(water100_oracle, mode):
    NN, scr, rows, ref = water100_oracle
    ctx = ctx_for(NN, scr, rows, "fp64", nuclear_sum=mode)
    ctx.initialize()
    K = ctx.download_K()
    scale = np.abs(ref.K).max()
    assert np.abs(K - ref.K).max() <= 1e-12 * scale


def test_potential_fp32_is_rounded_fp64(water100_oracle):
    NN, scr, rows, ref = water100_oracle
    ctx = ctx_for(NN, scr, rows, "mixed")
    ctx.initialize()
    K = np.asarray(ctx.download_K(), np.float32)
    want = ref.K.astype(np.float32)
    ulp = np.spacing(np.abs(want)).astype(np.float64)
    assert (np.abs(K.astype(np.float64) - want.astype(np.float64)) <= ulp).all()


@pytest.mark.parametrize("precision,mode", [("fp64", AUTO), ("mixed", AUTO), ("mixed", DIRECT)])
def test_hf_forces_match_oracle(water100_oracle, precision, mode):
    from realmolecule_b200 import _lib as L
    NN, scr, rows, ref = water100_oracle
    ctx = ctx_for(NN, scr, rows, precision, nuclear_sum=mode)
    ctx.initialize()
    psi = np.asarray(ctx.download(psi=True, label=False)["psi"], np.float64)
    F = ctx.forces(L.FORCE_HF)
    saved = ref.U.copy()
    try:
        ref.U[:] = psi.reshape(ref.U.shape)
        want = ref.forces()
    finally:
        ref.U[:] = saved
    nuc = [q for q, r in enumerate(rows) if r["Z_nuc"] > 0]
    scale = np.abs(want[nuc]).max()
    assert np.abs(F[nuc] - want[nuc]).max() <= 1e-10 * scale


def test_potential_full_size_samples():
    """The 1000-water geometry on its 320^3 grid: K at 4096 sampled interior points against an
    independent numpy sum over all 3000 nuclei (scipy's erf), 1e-12 relative."""
    from scipy.special import erf
    from realmolecule_b200 import configs as C
    g = C.water1000()
    rows = C.to_domain_atoms(g)
    ctx = ctx_for(g.NN, g.NN * g.h, rows, "fp64")
    ctx.initialize()
    K = ctx.download_K().reshape(g.NN + 1, g.NN + 1, g.NN + 1)
    rng = np.random.default_rng(7)
    ijk = rng.integers(1, g.NN, size=(4096, 3))
    nuc = np.array([[r["i"], r["j"], r["k"]] for r in rows if r["Z_nuc"] > 0]) * g.h
    Z = np.array([r["Z_nuc"] for r in rows if r["Z_nuc"] > 0])
    sigma = g.h
    x = ijk * g.h
    want = np.empty(len(x))
    for q in range(0, len(x), 256):
        d = x[q:q + 256, None, :] - nuc[None, :, :]
        r = np.sqrt((d * d).sum(-1))
        want[q:q + 256] = (Z * erf(r / (np.sqrt(2.0) * sigma)) / r).sum(-1)
    got = K[ijk[:, 0], ijk[:, 1], ijk[:, 2]]
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tiled_adjoint_matches_direct(precision):
    """One water on 128^3 at h = 0.3 (3 nuclei, tiles forced; the corner tiles see them as far):
    40 recorded steps from the same state; the adjoint forces and dE/dv through the tiled gather
    equal the direct gather's."""
    from realmolecule_b200 import configs as C
    g = C.h2o64()
    g.NN, g.h = 128, 0.3
    rows = C.to_domain_atoms(g)
    out = []
    for mode in (DIRECT, TILED):
        ctx = ctx_for(128, 128 * 0.3, rows, precision, nuclear_sum=mode, label_until=100)
        ctx.initialize()
        ctx.step(200)
        ctx.set_adjoint_window(40)
        ctx.step(40)
        F, dv = ctx.adjoint(forces=True, potential=True)
        out.append((F, np.asarray(dv)))
    (F0, d0), (F1, d1) = out
    assert np.abs(F1 - F0).max() <= 1e-10 * np.abs(F0).max()
    assert np.abs(d1 - d0).max() <= 1e-12 * np.abs(d0).max()
