"""A NaN uploaded into psi on the host is reported as RQ_ENONFINITE, never accepted silently.

The normalisation entry points read their error word back; the context and batch readouts
report a normalisation that met a NaN/Inf domain norm (the kernel leaves that domain unscaled).
The NaN is planted in host memory before the upload: the kernels only do IEEE arithmetic on it.
"""
import os
import sys

import numpy as np
import pytest

from gpu_util import dev, host, ptr, stream

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _state(NN=32, n_atoms=6, seed=21):
    sys.path.insert(0, GOLD)
    from make_golden import seeded_state
    return seeded_state(NN, n_atoms, seed)


def test_kernel_normalize_reports_nan_norm_and_scales_other_domains():
    from realmolecule_b200 import _lib
    lib = _lib.load()
    NN, nA = 32, 6
    S = NN + 1
    st = _state(NN, nA)
    U = st["U"].copy()
    lab = st["label"]
    bad = int(np.flatnonzero((lab == 2) & (U > 0))[0])
    U[bad] = np.nan
    Z = dev(st["atoms5"].reshape(nA, 5)[:, 3].copy())
    L = dev(lab)
    h3 = np.float32(0.25 ** 3)
    for noalloc in (False, True):
        Ud = dev(U)
        if noalloc:
            rc = lib.rq_kernel_normalize_sp_noalloc(ptr(Ud), ptr(L), ptr(Z), nA, S, h3, stream())
        else:
            rc = lib.rq_kernel_normalize_sp(ptr(Ud), ptr(L), ptr(Z), nA, S, h3, None, stream())
        assert rc == _lib.RQ_ENONFINITE
        out = host(Ud)
        # the NaN domain is left as it was; every other domain is normalised to its charge
        assert np.array_equal(out[lab == 2][np.isfinite(U[lab == 2])], U[lab == 2][np.isfinite(U[lab == 2])])
        for d in (0, 1, 3):
            n = float(np.sum(out[lab == d].astype(np.float64) ** 2) * float(h3))
            assert abs(n - float(st["atoms5"][d * 5 + 3])) < 1e-4 * n


@pytest.mark.parametrize("flavor", ["solver.py", "new"])
def test_context_energy_reports_nan_psi(flavor):
    from realmolecule_b200 import Context, _lib as L, configs
    if flavor == "solver.py":
        cfg = {"gridN": 32, "screen": 8.0, "atoms": [
            {"i": 13, "j": 14, "k": 16, "Z": 1, "rc": 0}, {"i": 16, "j": 16, "k": 16, "Z": 2, "rc": 0.4},
            {"i": 19, "j": 14, "k": 16, "Z": 1, "rc": 0}]}
        ctx = Context(32, cfg["screen"], cfg["atoms"], flavor="solver.py")
        steps = 20  # one normalisation
    else:
        g = configs.h2o64()
        g.NN, g.h = 32, 0.5
        ctx = Context(g.NN, g.screen, configs.to_domain_atoms(g), flavor="new", precision="mixed")
        steps = 4  # one normalisation
    ctx.initialize()
    st = ctx.download(psi=True, label=True)
    psi = st["psi"].copy()
    q = int(np.argmax(psi))
    psi[q] = np.nan
    ctx.upload(psi=psi)
    ctx.step(steps)
    with pytest.raises(L.RqError) as e:
        ctx.energy()
    assert e.value.status == L.RQ_ENONFINITE
    ctx.close()
