"""The mol_fast.js multi-field solver (rq_mf_*) on the GPU against the oracle's restatement
(oracle.MolFastDriver over orc_mf_*).

Both sides run the shaders' f32 operations in the reference's order and the reduction keeps the
reference's workgroup trees, so after a frame every field, every f32 sum, the forces, the slice
buffer and K are bit-equal.  The initial state is built in FP64 on both sides; there the sums of
the pre-normalisation run in another order and CUDA's exp may differ from the host's in the last
bit of an f64, so that comparison allows one f32 ulp on a small fraction of the values.  The
frame tests start both sides from the oracle's initial state.
"""
import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu

H2 = dict(nuclei=[{"i": 14, "j": 16, "k": 16, "Z": 1}, {"i": 18, "j": 16, "k": 16, "Z": 1}], NN=32, screen=8.0)
# multi-occupancy (selfN > 1), rc cusps, tilt, external field, Pauli and Thomas-Fermi terms
LIH = dict(nuclei=[{"i": 15, "j": 18, "k": 17, "Z": 3, "rc": 0.6, "z_init": 2.5, "tilt_y": 0.01},
                   {"i": 22, "j": 17.5, "k": 18, "Z": 1, "tilt_x": -0.02},
                   {"i": 12.25, "j": 18, "k": 17, "Z": 0, "z_init": 1.2}],
           NN=36, screen=9.0, norm_targets=[2, 1, 1], kc_multi=1.5, beta_pauli=0.05, field_x=0.01,
           alpha_tf=0.2)
# SHELL_MODE: per-orbital rc / r_out (released mid-run), hemi / third / tetra / hemi_third splits,
# split siblings sharing their Hartree subtraction
SPLIT = dict(nuclei=[{"i": 18, "j": 18, "k": 18, "Z": 2, "rc": 0.5, "split": "hemi", "split_idx": 0,
                      "split_axis": [1, 1, 0]},
                     {"i": 18, "j": 18, "k": 18, "Z": 2, "rc": 0.5, "split": "hemi", "split_idx": 1,
                      "split_axis": [1, 1, 0]},
                     {"i": 18, "j": 18, "k": 18, "Z": 1, "r_out": 2.0, "split": "third", "split_idx": 2,
                      "split_axis": [0, 0, 1]},
                     {"i": 18, "j": 18, "k": 18, "Z": 1, "split": "tetra", "split_idx": 1},
                     {"i": 23, "j": 18, "k": 18, "Z": 1, "split": "hemi_third", "split_idx": 2,
                      "split_axis": [0.3, 0.2, 1.0]},
                     {"i": 13, "j": 19, "k": 18, "Z": 1, "split": "hemi_third", "split_idx": 0, "split_fix": False}],
             NN=36, screen=9.0, shell_mode=True, r_out_release_step=40)

CASES = [("h2", H2, 70, 25), ("lih_terms", LIH, 60, 20), ("shell_splits", SPLIT, 50, 25)]


def pair(cfg, vcycle_interval):
    from realmolecule_b200.mol_fast import MolFast
    kw = {k: v for k, v in cfg.items() if k != "nuclei"}
    ref = orc.MolFastDriver(cfg["nuclei"], vcycle_interval=vcycle_interval, **kw)
    ref.initialize()
    gpu = MolFast(cfg["nuclei"], vcycle_interval=vcycle_interval, **kw)
    return ref, gpu


def same(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_initial_state(case):
    _, cfg, _, vi = case
    ref, gpu = pair(cfg, vi)
    assert same(gpu.K(), ref.K)
    for m in range(gpu.n):
        g, r = gpu.fields(m), ref.fields(m)
        for key in ("U", "W", "P"):
            eq = (g[key].view(np.uint32) == r[key].view(np.uint32)).mean()
            assert eq >= 0.9999, (m, key, eq)
            ulps = np.abs(g[key].view(np.int32).astype(np.int64) - r[key].view(np.int32).astype(np.int64))
            assert ulps.max() <= 1, (m, key, ulps.max())
    gpu.close()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_frames_bit_exact(case):
    _, cfg, nsteps, vi = case
    ref, gpu = pair(cfg, vi)
    for m in range(gpu.n):
        f = ref.fields(m)
        gpu.set_fields(m, f["U"], f["W"], f["P"])
    # two frames of different lengths: frame-local normalisation and V-cycle counters
    for n in (nsteps, 33):
        ref.do_steps(n)
        out = gpu.doSteps(n)
        assert same(gpu.sums, ref.sums), (n, gpu.sums, ref.sums)
        assert out["E"] == ref.E and out["dipole"] == ref.dipole
    for m in range(gpu.n):
        g, r = gpu.fields(m), ref.fields(m)
        for key in ("U", "W", "P"):
            assert same(g[key], r[key]), (m, key)
    fd = ref.compute_forces()
    gpu.computeForces()
    assert gpu.nuc_force == ref.force
    assert same(gpu.extract(), ref.extract())
    assert gpu.kernel_launches > 0
    gpu.close()


def test_dynamics_frames_move_nuclei_like_the_page():
    cfg = dict(H2, nuclei=[{"i": 14.5, "j": 16, "k": 16, "Z": 1}, {"i": 18, "j": 16.25, "k": 16, "Z": 1}])
    ref, gpu = pair(cfg, 50)
    for m in range(gpu.n):
        f = ref.fields(m)
        gpu.set_fields(m, f["U"], f["W"], f["P"])
    gpu.dt_nuc = ref.dt_nuc = 40.0
    for _ in range(3):
        ref.do_steps(60)
        ref.compute_forces()
        moved = ref.step_nuclei()
        gpu.doSteps(60)
        gpu.computeForces()
        assert gpu.stepNuclei() == moved
        assert [(a["i"], a["j"], a["k"]) for a in gpu.nuclei] == [(a["i"], a["j"], a["k"]) for a in ref.nuclei]
        assert same(gpu.K(), ref.K)
        assert gpu.E_KK == ref.E_KK
    assert moved
    for m in range(gpu.n):
        assert same(gpu.fields(m)["U"], ref.fields(m)["U"])
    gpu.close()


def test_invalid_configs_are_errors():
    from realmolecule_b200 import _lib as L
    from realmolecule_b200.mol_fast import MolFast
    with pytest.raises(ValueError):
        MolFast(H2["nuclei"], NN=33)
    with pytest.raises(L.RqError):
        MolFast(H2["nuclei"], NN=32, vcycle_interval=0)
