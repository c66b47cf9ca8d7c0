"""The oracle (oracle/rq_oracle.c) pinned against the reference's own outputs (CPU only).

Golden vectors come from tests/golden/make_golden.py, which ran the reference's
cloud/solver.py kernel text compiled for the host and the untouched RealQMSolver class.
"""
import json
import os

import numpy as np
import pytest

import oracle as orc

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def g():
    return dict(np.load(os.path.join(GOLD, "solverpy_kernels_nn16.npz")))


def test_update_bit_exact(g):
    S = int(g["NN"]) + 1
    out = np.zeros_like(g["in_U"])
    orc.O().sp_update(g["in_U"], out, g["in_K"], g["in_P"], g["in_label"], S, g["half_dv"], g["dtv"])
    assert np.array_equal(out.view(np.uint32), g["out_updateU"].view(np.uint32))


def test_jacobi_bit_exact(g):
    S = int(g["NN"]) + 1
    h = float(g["h"])
    out = np.zeros_like(g["in_P"])
    orc.O().sp_jacobi(g["in_P"], out, g["in_U"], S, np.float32(h * h), np.float32(2 * np.pi))
    assert np.array_equal(out.view(np.uint32), g["out_jacobiStep"].view(np.uint32))


def test_init_trial_and_K_bit_exact(g):
    S = int(g["NN"]) + 1
    h = np.float32(g["h"])
    S3 = S ** 3
    U, K, best = (np.zeros(S3, np.float32) for _ in range(3))
    lab = np.zeros(S3, np.int32)
    orc.O().sp_init_trial(U, lab, K, best, g["in_atoms5"], int(g["nAtoms"]), S, h, np.float32(h * h))
    assert np.array_equal(U.view(np.uint32), g["out_initTrial_U"].view(np.uint32))
    assert np.array_equal(K.view(np.uint32), g["out_initTrial_K"].view(np.uint32))
    assert np.array_equal(lab, g["out_initTrial_label"])
    K2 = np.zeros(S3, np.float32)
    orc.O().sp_recompute_K(K2, g["in_atoms5"], int(g["nAtoms"]), S, h, np.float32(h * h))
    assert np.array_equal(K2.view(np.uint32), g["out_recomputeK"].view(np.uint32))


def test_labels_inplace_matches_reference(g):
    """The decision rule, pinned against the reference kernel run serially in place."""
    S = int(g["NN"]) + 1
    h = np.float32(g["h"])
    lab = g["in_label"].copy()
    orc.O().sp_boundary_inplace_lex(lab, g["in_atoms5"], int(g["nAtoms"]), S, h, np.float32(h * h))
    assert np.array_equal(lab, g["out_boundaryEvolve_inplace"])


def test_labels_snapshot_differs_only_by_cascade(g):
    """Snapshot semantics (the CUDA kernel's) equal the in-place result wherever no
    already-updated neighbour was read (first sweep of the lexicographic order)."""
    S = int(g["NN"]) + 1
    h = np.float32(g["h"])
    snap = np.zeros_like(g["in_label"])
    orc.O().sp_boundary_snapshot(g["in_label"], snap, g["in_atoms5"], int(g["nAtoms"]), S, h, np.float32(h * h))
    changed = snap != g["in_label"]
    assert changed.sum() > 0
    # cells whose in-place and snapshot results differ must have a neighbour that flipped earlier
    ref = g["out_boundaryEvolve_inplace"]
    diff = np.flatnonzero(snap != ref)
    flipped = ref != g["in_label"]
    S2 = S * S
    for idx in diff:
        assert flipped[idx - 1] or flipped[idx - S] or flipped[idx - S2]


def test_forces_match_reference(g):
    S = int(g["NN"]) + 1
    h = np.float32(g["h"])
    F = np.zeros(int(g["nAtoms"]) * 3, np.float64)
    orc.O().sp_forces(g["in_U"], g["in_atoms5"], int(g["nAtoms"]), S, h, np.float32(h * h), np.float32(h ** 3), F)
    np.testing.assert_allclose(F, g["out_computeForceAll"], rtol=2e-5, atol=1e-6)


def test_normalize_matches_reference(g):
    S = int(g["NN"]) + 1
    nA = int(g["nAtoms"])
    h3 = np.float32(float(g["h"]) ** 3)
    norms = np.zeros(nA, np.float32)
    orc.O().sp_norms_f32_seq(g["in_U"], g["in_label"], S ** 3, nA, h3, norms)
    assert np.array_equal(norms.view(np.uint32), g["norms_f32"].view(np.uint32))
    U = g["in_U"].copy()
    Z = g["in_atoms5"].reshape(nA, 5)[:, 3].copy()
    orc.O().sp_normalize(U, g["in_label"], norms, Z, S ** 3, nA)
    assert np.array_equal(U.view(np.uint32), g["out_normalizeU"].view(np.uint32))


def test_driver_matches_reference_run():
    """200 steps of the restated schedule (FP64 norms) against the untouched reference
    RealQMSolver (serial kernels, in-place labels)."""
    with open(os.path.join(GOLD, "solverpy_run_h2o_nn32.json")) as f:
        gold = json.load(f)
    d = orc.SolverPyDriver(gold["config"], kernels="oracle", label_mode="inplace_lex")
    d.initialize()
    d.run(gold["steps"])
    d.energy()
    last = gold["snapshots"][-1]
    for k, v in (("E_T", d.E_T), ("E_eK", d.E_eK), ("E_ee", d.E_ee), ("E_KK", d.E_KK)):
        assert abs(v - last[k]) < 2e-5 * max(1.0, abs(last[k])), (k, v, last[k])
    assert int(np.asarray(d.label, np.int64).sum()) == gold["final_label_checksum"]


def test_hairpin_fixture_shape():
    with open(os.path.join(GOLD, "hairpin_config.json")) as f:
        cfg = json.load(f)
    assert cfg["gridN"] == 300 and len(cfg["atoms"]) == 267 and cfg["nProtein"] == 87
    with open(os.path.join(GOLD, "hairpin_golden.json")) as f:
        gold = json.load(f)
    assert [s["step"] for s in gold["snapshots"]] == list(range(1000, 10001, 1000))
