"""The realqm_rb.js red-black multi-field solver (rq_rb_*) on the GPU against the oracle's
restatement (oracle.RealqmRbDriver, the reference's sequential per-electron passes).

Red-black passes, norm reductions and scales run the reference's f32 operations in its order,
so after frames every field and the slice buffer are bit-equal; the energies are FP64 sums in
another order (1e-12 relative).  The initial u is exp evaluated in f64 and rounded to f32 on
both sides; the device and host f64 exp may differ in the last bit, so that one comparison
allows one f32 ulp on a small fraction of values.  Frame tests start both sides from the
oracle's initial state.
"""
import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu

H2 = dict(nuclei=[{"i": 12, "j": 16, "k": 16, "Z": 1, "rc": 0, "ne": 1},
                  {"i": 20, "j": 16, "k": 16, "Z": 1, "rc": 0, "ne": 1}], NN=32, screen=8.0)
# a two-electron nucleus split into halves at the box centre, an r_c exclusion mask and a front cut
HEH = dict(nuclei=[{"i": 16, "j": 16, "k": 16, "Z": 2, "rc": 0.8, "ne": 2, "rc_excl": 0.35},
                   {"i": 23, "j": 15, "k": 16, "Z": 1, "rc": 0.8, "ne": 1}], NN=32, screen=8.0,
           norm_targets=[1, 1, 1])
# an occupation above 1 (the (n-1)/n self term), a fractional position (its mask marks nothing)
LI3 = dict(nuclei=[{"i": 14, "j": 14, "k": 15, "Z": 3, "rc": 0.6, "ne": 1, "rc_excl": 0.3},
                   {"i": 20.5, "j": 17, "k": 15, "Z": 1, "ne": 1, "rc_excl": 0.3},
                   {"i": 15, "j": 21, "k": 16, "Z": 1, "ne": 1}], NN=34, screen=8.5, norm_targets=[2, 1, 1])

CASES = [("h2", H2), ("heh_split_mask", HEH), ("occupation_two", LI3)]


def pair(cfg):
    from realmolecule_b200.realqm_rb import RealqmRb
    kw = {k: v for k, v in cfg.items() if k != "nuclei"}
    ref = orc.RealqmRbDriver(cfg["nuclei"], **kw)
    ref.initialize()
    gpu = RealqmRb(cfg["nuclei"], **kw)
    return ref, gpu


def same(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_initial_state(case):
    ref, gpu = pair(case[1])
    assert same(gpu.K(), ref.K)
    for m in range(gpu.nelec):
        g, r = gpu.fields(m), ref.fields(m)
        assert same(g["W"], r["W"]) and same(g["P"], r["P"]), m
        eq = (g["U"].view(np.uint32) == r["U"].view(np.uint32)).mean()
        ulps = np.abs(g["U"].view(np.int32).astype(np.int64) - r["U"].view(np.int32).astype(np.int64))
        assert eq >= 0.9999 and ulps.max() <= 1, (m, eq, ulps.max())
    gpu.close()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_frames_bit_exact(case):
    ref, gpu = pair(case[1])
    for m in range(gpu.nelec):
        f = ref.fields(m)
        gpu.set_fields(m, f["U"], f["W"], f["P"])
    for n in (7, 12):  # frame-local normalisation at steps 0 and 5 of each frame
        ref.do_steps(n)
        gpu.doSteps(n)
    for m in range(gpu.nelec):
        g, r = gpu.fields(m), ref.fields(m)
        for key in ("U", "W", "P"):
            assert same(g[key], r[key]), (m, key)
    e = gpu.computeEnergy()
    er = ref.energy()
    for a, b in zip((e["E_T"], e["E_eK"], e["E_ee"]), er):
        assert abs(a - b) <= 1e-12 * max(1.0, abs(b)), (a, b)
    assert same(gpu.extractSlice(), ref.slice())
    assert gpu.kernel_launches > 0
    gpu.close()


def test_page_frames_and_errors():
    from realmolecule_b200.realqm_rb import RealqmRb
    g = RealqmRb.from_page({"USER_NN": 24, "USER_SCREEN": 6, "USER_D": 6, "USER_STEPS": 30})
    assert [a["i"] for a in g.nuclei] == [9, 15]
    out = None
    for _ in range(4):
        out = g.frame()
    assert out["stepCount"] == 30 and out["done"] and np.isfinite(out["E_tot"])
    g.close()
    with pytest.raises(ValueError):
        RealqmRb(H2["nuclei"], NN=32, screen=8.0, nelec=3)
