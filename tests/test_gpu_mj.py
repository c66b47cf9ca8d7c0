"""molecule.js flavour on the GPU against the oracle's restatement of doSteps.

From an identical state (the oracle's initial psi and labels uploaded through the C ABI) whole
frames -- weighted Jacobi, the 2-level V-cycle, the update with r_c exclusion, the u32
fixed-point normalisation and the level-set label passes -- must agree BIT FOR BIT (every
operation is strict f32 in the reference's order and the norms are integer sums).  The
initial trial state itself goes through expf (CUDA vs libm): K is bit-exact, psi within 2 ulp.
"""
import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu


def atoms_case(kind):
    if kind == "water":  # molecule.js idiom: O with a pseudopotential core, two bare-Coulomb H
        return 40, 10.0, [{"i": 20, "j": 20, "k": 20, "Z": 6, "Z_nuc": 6, "rc": 0.4},
                          {"i": 23, "j": 17, "k": 20, "Z": 1, "Z_nuc": 1, "rc": 0.0},
                          {"i": 17, "j": 17, "k": 20, "Z": 1, "Z_nuc": 1, "rc": 0.0}]
    if kind == "bare":  # a bare proton (Z=0, Z_nuc>0, rc>0) switches on the bare-nuclei exclusion
        return 32, 8.0, [{"i": 14, "j": 16, "k": 16, "Z": 2, "Z_nuc": 2, "rc": 0.3},
                         {"i": 19, "j": 16, "k": 16, "Z": 1, "Z_nuc": 1, "rc": 0.0},
                         {"i": 16, "j": 20, "k": 16, "Z": 0, "Z_nuc": 1, "rc": 0.3},
                         {"i": 16, "j": 12, "k": 14, "Z": 1, "Z_nuc": 1, "rc": 0.0}]
    if kind == "ten":  # 10 domains: the self-interaction correction runs every frame (NELEC <= 15)
        rng = np.random.default_rng(11)
        rows = []
        for n in range(10):
            p = rng.integers(12, 28, 3)
            z = float(rng.integers(1, 3))
            rows.append({"i": int(p[0]), "j": int(p[1]), "k": int(p[2]), "Z": z, "Z_nuc": z,
                         "rc": float(rng.choice([0.0, 0.35]))})
        return 40, 10.0, rows
    rng = np.random.default_rng(3)  # many domains
    rows = []
    for n in range(24):
        p = rng.integers(10, 38, 3)
        rows.append({"i": int(p[0]), "j": int(p[1]), "k": int(p[2]), "Z": float(rng.integers(1, 3)),
                     "Z_nuc": 0.0, "rc": float(rng.choice([0.0, 0.35]))})
        rows[-1]["Z_nuc"] = rows[-1]["Z"]
    return 48, 12.0, rows


def make_pair(kind, **opts):
    from realmolecule_b200 import Context
    NN, screen, rows = atoms_case(kind)
    ref = orc.MoleculeJsDriver(NN, screen, rows, **opts)
    ref.initialize()
    ctx = Context(NN, screen, rows, flavor="molecule.js", **{k: v for k, v in opts.items() if v is not None})
    ctx.initialize()
    return ref, ctx


@pytest.mark.parametrize("kind", ["water", "bare", "many"])
def test_init_K_bit_exact_psi_close(kind):
    ref, ctx = make_pair(kind)
    assert np.array_equal(ctx.download_K().view(np.uint32), ref.K.view(np.uint32))
    st = ctx.download(psi=True, label=True)
    np.testing.assert_allclose(st["psi"], ref.U, rtol=3e-7, atol=0)
    bad = np.flatnonzero(st["label"] != ref.label.astype(np.int32))
    assert bad.size <= 3


@pytest.mark.parametrize("kind", ["water", "bare", "many"])
def test_frames_bit_exact(kind):
    opts = dict(steps_per_frame=7, norm_interval=5, vcycle_interval=3)
    ref, ctx = make_pair(kind, **opts)
    ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    lab0 = ref.label.copy()
    nsteps = 3 * 7 + 2
    for _ in range(nsteps):
        ref.step()
    ctx.step(nsteps)
    st = ctx.download(psi=True, label=True, W=True, P=True)
    assert np.array_equal(st["label"], ref.label.astype(np.int32))
    assert np.array_equal(st["W"].view(np.uint32), ref.W.view(np.uint32))
    assert np.array_equal(st["P"].view(np.uint32), ref.P.view(np.uint32))
    assert np.array_equal(st["psi"].view(np.uint32), ref.U.view(np.uint32))
    assert (ref.label != lab0).sum() > 0 or kind == "water"  # the level set moved somewhere


def test_energy_and_dipole_sums():
    from realmolecule_b200 import _lib as L
    ref, ctx = make_pair("many", steps_per_frame=5)
    ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    for _ in range(10):
        ref.step()
    ctx.step(10)
    e, pd = ctx.energy(per_domain=True)
    o = ref.energy()
    nH = sum(1 for a in ref.rows if a["Z"] == 1 and a.get("rc", 0) == 0)
    raw = {100: (0.5, -1.0), 300: (0.5, -1.0)}.get(ref.NN, (0.503, -1.028))
    T = e[L.E_T] - nH * (0.5 - raw[0])
    EK = e[L.E_EK] - nH * (-1.0 - raw[1])
    np.testing.assert_allclose([T, EK, e[L.E_EE]], o[:3], rtol=1e-9)
    nuc = np.zeros(3)
    for a in ref.rows:
        if a["Z"] != 0:
            nuc += a["Z"] * np.array([a["i"], a["j"], a["k"]], float) * ref.hd
    np.testing.assert_allclose([e[L.E_DIPX], e[L.E_DIPY], e[L.E_DIPZ]], nuc - o[3:], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(pd[:, 1].sum(), T, rtol=1e-12)


def test_forces_gradp_and_hf():
    from realmolecule_b200 import _lib as L
    ref, ctx = make_pair("water", steps_per_frame=5)
    ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    for _ in range(10):
        ref.step()
    ctx.step(10)
    R = max(5, round(3.0 / ref.hd))
    Fo = np.zeros(ref.nA * 3)
    orc.O().mj_force_gradP(ref.P, orc.C.addressof(ref.atoms), ref.nA, ref.S, np.float32(1 / ref.hd), R, Fo)
    Fg = ctx.forces(L.FORCE_GRADP)
    np.testing.assert_allclose(Fg.reshape(-1), Fo, rtol=1e-9, atol=1e-12)
    Fo2 = np.zeros(ref.nA * 3)
    orc.O().mj_force_hf(ref.U, orc.C.addressof(ref.atoms), ref.nA, ref.S, ref.h, ref.h2, Fo2)
    Fh = ctx.forces(L.FORCE_HF)
    np.testing.assert_allclose(Fh.reshape(-1), Fo2, rtol=2e-4, atol=1e-5 * np.abs(Fo2).max())


def test_set_atoms_persistent_relabel():
    ref, ctx = make_pair("water", steps_per_frame=5)
    ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    rows = [dict(a) for a in ref.rows]
    rows[1]["i"] += 2.7  # truncated to +2 cells on the GPU like the Uint32Array store
    rows[2]["j"] -= 1.2
    ref.set_positions(rows)
    ctx.set_atoms(rows)
    assert np.array_equal(ctx.download_K().view(np.uint32), ref.K.view(np.uint32))
    lab = ctx.download(psi=False, label=True)["label"]
    # bestU came from each side's own init (expf), so allow a handful of near-tie cells
    assert (lab != ref.label.astype(np.int32)).sum() <= 5


@pytest.mark.parametrize("kind,frames", [("ten", 3), ("many", 6)])
def test_frames_with_self_interaction_correction_bit_exact(kind, frames):
    """cfg.sic: on the reference's frames (every frame for NELEC <= 15, every 5th for <= 30, never
    on frame 0) each domain's own potential is solved (4 sweeps, the coarse correction, 4 sweeps)
    and P_m / Z_m leaves Pother on the domain -- bit for bit with the oracle, through the graphs
    of whole SIC periods."""
    opts = dict(steps_per_frame=7, norm_interval=5, vcycle_interval=3)
    from realmolecule_b200 import Context
    NN, screen, rows = atoms_case(kind)
    ref = orc.MoleculeJsDriver(NN, screen, rows, sic=True, **opts)
    ref.initialize()
    ctx = Context(NN, screen, rows, flavor="molecule.js", sic=1, **opts)
    ctx.initialize()
    ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    nsteps = frames * 7 + 2
    plain = orc.MoleculeJsDriver(NN, screen, rows, **opts)  # the same run without the correction
    plain.initialize()
    plain.U[:] = ref.U
    for _ in range(nsteps):
        ref.step()
        plain.step()
    ctx.step(nsteps)
    st = ctx.download(psi=True, label=True, W=True, P=True)
    assert not np.array_equal(ref.Pother, plain.Pother)  # the correction did run
    assert np.array_equal(st["label"], ref.label.astype(np.int32))
    assert np.array_equal(st["W"].view(np.uint32), ref.W.view(np.uint32))
    assert np.array_equal(st["P"].view(np.uint32), ref.P.view(np.uint32))
    assert np.array_equal(st["psi"].view(np.uint32), ref.U.view(np.uint32))
    from realmolecule_b200 import _lib as L
    e = ctx.energy()
    np.testing.assert_allclose(e[L.E_EE], ref.energy()[2], rtol=1e-9)  # V_ee reads the corrected Pother


@pytest.mark.parametrize("kind", ["water", "bare"])
def test_direct_per_electron_poisson_bit_exact(kind):
    """cfg.sic with NELEC <= 5: the reference's direct path -- a persistent P_m per domain,
    initialised to sum_{n != m} 0.5/r and relaxed by 10 Jacobi sweeps on the density of the other
    domains every step, copied into Pother on domain m -- bit for bit with the oracle, and the
    gradP force reads that Pother."""
    from realmolecule_b200 import Context, _lib as L
    opts = dict(steps_per_frame=7, norm_interval=5, vcycle_interval=3)
    NN, screen, rows = atoms_case(kind)
    ref = orc.MoleculeJsDriver(NN, screen, rows, sic=True, **opts)
    ref.initialize()
    assert ref.direct
    ctx = Context(NN, screen, rows, flavor="molecule.js", sic=1, **opts)
    ctx.initialize()
    ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    nsteps = 2 * 7 + 3
    for _ in range(nsteps):
        ref.step()
    ctx.step(nsteps)
    st = ctx.download(psi=True, label=True, W=True)
    assert np.array_equal(st["label"], ref.label.astype(np.int32))
    assert np.array_equal(st["W"].view(np.uint32), ref.W.view(np.uint32))
    assert np.array_equal(st["psi"].view(np.uint32), ref.U.view(np.uint32))
    np.testing.assert_allclose(ctx.energy()[L.E_EE], ref.energy()[2], rtol=1e-9)
    R = max(5, round(3.0 / ref.hd))
    Fo = np.zeros(ref.nA * 3)
    orc.O().mj_force_gradP(ref.Pother, orc.C.addressof(ref.atoms), ref.nA, ref.S, np.float32(1 / ref.hd), R, Fo)
    np.testing.assert_allclose(ctx.forces(L.FORCE_GRADP).reshape(-1), Fo, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("kind", ["water", "ten"])
def test_frames_with_chebyshev_bit_exact(kind):
    """The Chebyshev update (molecule.js:345-421) with the page's omega recurrence fed by each
    frame's energy (both sides form E from FP64 sums; omega is rounded to f32 before use)."""
    from realmolecule_b200 import Context
    NN, screen, rows = atoms_case(kind)
    ref = orc.MoleculeJsDriver(NN, screen, rows, steps_per_frame=10, chebyshev=True)
    ref.initialize()
    ctx = Context(NN, screen, rows, flavor="molecule.js", steps_per_frame=10, chebyshev=1)
    ctx.initialize()
    ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    for _ in range(30):  # three frames: omega 1, then the recurrence with E of frames 1 and 2
        ref.step()
    ctx.step(30)
    st = ctx.download(psi=True, label=True, W=True, P=True)
    assert np.array_equal(st["psi"].view(np.uint32), ref.U.view(np.uint32))
    assert np.array_equal(st["label"], ref.label.astype(np.int32))
    assert np.array_equal(st["W"].view(np.uint32), ref.W.view(np.uint32))
    assert ref.cheb_state > 1.01


def test_chebyshev_is_refused_with_bare_nuclei():
    from realmolecule_b200 import Context, _lib as L
    NN, screen, rows = atoms_case("bare")
    with pytest.raises(L.RqError) as e:
        Context(NN, screen, rows, flavor="molecule.js", chebyshev=1)
    assert e.value.status == L.RQ_ENOTSUP


@pytest.mark.parametrize("kind,sic", [("water", False), ("bare", False), ("water", True), ("ten", True),
                                      ("many", False)],
                         ids=["water", "bare_nuclei", "water_direct_poisson", "ten_sic", "many"])
def test_lobpcg_frames_bit_exact(kind, sic):
    """LOBPCG frames (doLOBPCGStep, molecule.js:3323-3740): the Poisson solve and Pother, 10
    iterations per domain with the inner products in the shaders' workgroup trees and the Ritz
    problems in the page's FP64 arithmetic (one device thread here), normalisation, one ITP
    update, the level-set passes.  Three frames: the first without a search direction (eager),
    the second captured into a CUDA graph, the third replayed from it."""
    from realmolecule_b200 import Context
    NN, screen, rows = atoms_case(kind)
    ref = orc.MoleculeJsDriver(NN, screen, rows, steps_per_frame=5, sic=sic, lobpcg=True)
    ref.initialize()
    ctx = Context(NN, screen, rows, flavor="molecule.js", steps_per_frame=5, sic=int(sic), lobpcg=1)
    ctx.initialize()
    ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    for _ in range(3):
        ref.step()
    ctx.step(3)
    st = ctx.download(psi=True, label=True, W=True, P=True)
    assert np.array_equal(st["psi"].view(np.uint32), ref.U.view(np.uint32))
    assert np.array_equal(st["label"] & 0x3FFFFFFF, ref.label.astype(np.int32))
    assert np.array_equal(st["W"].view(np.uint32), ref.W.view(np.uint32))
    assert np.array_equal(st["P"].view(np.uint32), ref.P.view(np.uint32))
    assert ref.frame == 3


@pytest.mark.parametrize("kind,groups", [("water", [[0, 1]]), ("many", [[0, 3, 5], [1, 2], [7, 9, 11, 13]])],
                         ids=["water", "many"])
def test_locked_groups_frames_bit_exact(kind, groups):
    """USER_LOCKED_GROUPS (molecule.js:490-503): boundaries between labels of one group stay put
    (W = max(W, 0.5)); frames bit-exact against the restatement, and different from the frames
    without the groups."""
    from realmolecule_b200 import Context, _lib as L
    opts = dict(steps_per_frame=7, norm_interval=5, vcycle_interval=3)
    NN, screen, rows = atoms_case(kind)
    ref = orc.MoleculeJsDriver(NN, screen, rows, locked_groups=groups, **opts)
    ref.initialize()
    free = orc.MoleculeJsDriver(NN, screen, rows, **opts)
    free.initialize()
    ctx = Context(NN, screen, rows, flavor="molecule.js", **opts)
    ctx.initialize()
    ctx.set_locked_groups(groups)
    ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    for _ in range(3 * 7 + 2):
        ref.step()
        free.step()
    ctx.step(3 * 7 + 2)
    st = ctx.download(psi=True, label=True, W=True)
    assert np.array_equal(st["label"], ref.label.astype(np.int32))
    assert np.array_equal(st["W"].view(np.uint32), ref.W.view(np.uint32))
    assert np.array_equal(st["psi"].view(np.uint32), ref.U.view(np.uint32))
    assert not np.array_equal(ref.W, free.W)
    with pytest.raises(L.RqError):
        ctx.set_locked_groups([[0, len(rows)]])
    with pytest.raises(L.RqError) as e:
        ctx.set_locked_groups([[0]] * 65)
    assert e.value.status == L.RQ_ENOTSUP
    ctx.set_locked_groups([])



SPLIT_CASES = {
    # three O-site domains in 120-degree sectors about the molecular-plane normal, two H domains
    "third": ([{"i": 20, "j": 20, "k": 20, "Z": 1, "Z_nuc": 2}, {"i": 20, "j": 20, "k": 20, "Z": 1, "Z_nuc": 2},
               {"i": 20, "j": 20, "k": 20, "Z": 1, "Z_nuc": 2}, {"i": 23, "j": 17, "k": 20, "Z": 1, "Z_nuc": 1},
               {"i": 17, "j": 17, "k": 20, "Z": 1, "Z_nuc": 1}],
              [{"type": "third", "idx": q, "axis": (0.0, 0.1, 1.0), "rot": 0.35} for q in range(3)] + [None, None]),
    # a two-electron site split into half spaces along a tilted axis, next to a whole-sphere H
    "hemi": ([{"i": 19, "j": 20, "k": 20, "Z": 1, "Z_nuc": 1}, {"i": 19, "j": 20, "k": 20, "Z": 1, "Z_nuc": 1},
              {"i": 23, "j": 21, "k": 20, "Z": 1, "Z_nuc": 1}],
             [{"type": "hemi", "idx": 0, "axis": (1.0, 1.0, 0.2)}, {"type": 2, "idx": 1, "axis": (1.0, 1.0, 0.2)},
              None]),
}


@pytest.mark.parametrize("case", sorted(SPLIT_CASES))
def test_shell_split_frames_bit_exact(case):
    """Shell splits (USER_SPLIT_*, molecule.js:27-32; inSplitAtom :197-226): the trial labelling
    keeps each split entry to its sector, and the level-set step cancels flips into foreign sectors
    and hands cells that left their sector to a neighbour whose sector holds them (:514-533)."""
    from realmolecule_b200 import Context
    rows, splits = SPLIT_CASES[case]
    opts = dict(steps_per_frame=7, norm_interval=5, vcycle_interval=3)
    ref = orc.MoleculeJsDriver(40, 10.0, rows, splits=splits, **opts)
    ref.initialize()
    whole = orc.MoleculeJsDriver(40, 10.0, rows, **opts)
    whole.initialize()
    assert (ref.label != whole.label).sum() > 1000  # the sectors decide the initial labelling
    ctx = Context(40, 10.0, rows, flavor="molecule.js", **opts)
    ctx.set_splits(splits)
    ctx.initialize()
    lab0 = ctx.download(psi=False, label=True)["label"]
    assert (lab0 != ref.label.astype(np.int32)).sum() <= 3  # init psi goes through expf: near-ties only
    ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    for _ in range(3 * 7 + 2):
        ref.step()
    ctx.step(3 * 7 + 2)
    st = ctx.download(psi=True, label=True, W=True)
    assert np.array_equal(st["label"], ref.label.astype(np.int32))
    assert np.array_equal(st["W"].view(np.uint32), ref.W.view(np.uint32))
    assert np.array_equal(st["psi"].view(np.uint32), ref.U.view(np.uint32))



def face_mask(S):
    i, j, k = np.indices((S, S, S)).reshape(3, -1)
    return (i == 0) | (i == S - 1) | (j == 0) | (j == S - 1) | (k == 0) | (k == S - 1)


def test_restart_rebuilds_from_scratch_and_keeps_W_and_the_spare_faces():
    """rq_restart (the classical-MD backbone's full restart, molecule.js:4236-4286): K, psi and labels
    rebuilt from scratch at the moved positions, P cleared, W kept.  The rebuild writes labelBuf
    only; the next level-set pass copies label2Buf back over all cells (:3103), so the face labels
    return to those of the last full copy -- on the GPU as in the restatement."""
    from realmolecule_b200 import Context
    opts = dict(steps_per_frame=7, norm_interval=5, vcycle_interval=3)
    NN, screen, rows = atoms_case("many")
    ref = orc.MoleculeJsDriver(NN, screen, rows, **opts)
    ref.initialize()
    ctx = Context(NN, screen, rows, flavor="molecule.js", **opts)
    ctx.initialize()
    ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    faces = face_mask(NN + 1)
    faces0 = ref.label[faces].astype(np.int32)
    for _ in range(14):
        ref.step()
    ctx.step(14)
    W0 = ctx.download(psi=False, W=True)["W"]
    moved = [dict(a) for a in rows]
    for a in moved[:8]:
        a["i"] = max(2, a["i"] - 8)  # toward the i = 0 face
    ref.set_positions(moved)
    ref.restart()
    ctx.set_atoms(moved)
    ctx.restart()
    st = ctx.download(psi=True, label=True, W=True, P=True)
    assert np.array_equal(st["W"].view(np.uint32), W0.view(np.uint32))
    assert not st["P"].any()
    assert np.array_equal(ctx.download_K().view(np.uint32), ref.K.view(np.uint32))
    assert (st["label"] != ref.label.astype(np.int32)).sum() <= 3  # trial psi through expf: near-ties
    np.testing.assert_allclose(st["psi"], ref.U, rtol=3e-7, atol=0)
    assert not np.array_equal(st["label"][faces], faces0)  # the rebuild relabelled face cells
    for _ in range(7):
        ref.step()
    ctx.step(7)
    lab = ctx.download(psi=False, label=True)["label"]
    assert np.array_equal(ref.label[faces].astype(np.int32), faces0)
    assert np.array_equal(lab[faces], faces0)



def test_freeze_boundary_then_release_bit_exact():
    """FREEZE_BOUNDARY (molecule.js:3095): frozen frames keep labels and W; after the release the
    level set moves again.  Frozen and released periods both run from CUDA graphs."""
    from realmolecule_b200 import Context
    opts = dict(steps_per_frame=7, norm_interval=5, vcycle_interval=3)
    NN, screen, rows = atoms_case("many")
    ref = orc.MoleculeJsDriver(NN, screen, rows, **opts)
    ref.initialize()
    ref.freeze = True
    ctx = Context(NN, screen, rows, flavor="molecule.js", **opts)
    ctx.initialize()
    ctx.set_freeze_boundary(True)
    ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    lab0, W0 = ref.label.copy(), ref.W.copy()
    for _ in range(21):
        ref.step()
    ctx.step(21)
    st = ctx.download(psi=True, label=True, W=True)
    assert np.array_equal(ref.label, lab0) and np.array_equal(ref.W, W0)
    assert np.array_equal(st["label"], lab0.astype(np.int32))
    assert np.array_equal(st["W"].view(np.uint32), W0.view(np.uint32))
    assert np.array_equal(st["psi"].view(np.uint32), ref.U.view(np.uint32))
    ref.freeze = False
    ctx.set_freeze_boundary(False)
    for _ in range(21):
        ref.step()
    ctx.step(21)
    st = ctx.download(psi=True, label=True, W=True)
    assert not np.array_equal(ref.label, lab0)
    assert np.array_equal(st["label"], ref.label.astype(np.int32))
    assert np.array_equal(st["W"].view(np.uint32), ref.W.view(np.uint32))
    assert np.array_equal(st["psi"].view(np.uint32), ref.U.view(np.uint32))


@pytest.mark.parametrize("kind", ["water", "bare"])
def test_init_positions(kind):
    """window.USER_INIT_POS (molecule.js:1905-1981): trial psi and labels from the atoms moved to
    their init positions (k kept), K rebuilt by recomputeK at the true positions -- K bit-exact,
    psi within 2 ulp, labels up to near-ties; then frames from the uploaded state bit-exact."""
    from realmolecule_b200 import Context
    NN, screen, rows = atoms_case(kind)
    init = [(r["i"] + 2, r["j"] - 1) if q % 2 == 0 else None for q, r in enumerate(rows)]
    opts = dict(steps_per_frame=7, norm_interval=5, vcycle_interval=3)
    ref = orc.MoleculeJsDriver(NN, screen, rows, **opts)
    ref.initialize(init_pos=init)
    plain = orc.MoleculeJsDriver(NN, screen, rows, **opts)
    plain.initialize()
    assert (ref.label != plain.label).sum() > 100  # the moved trial psi changes the labels
    ctx = Context(NN, screen, rows, flavor="molecule.js", **opts)
    ctx.set_init_positions(init)
    ctx.initialize()
    assert np.array_equal(ctx.download_K().view(np.uint32), ref.K.view(np.uint32))
    st = ctx.download(psi=True, label=True)
    np.testing.assert_allclose(st["psi"], ref.U, rtol=3e-7, atol=0)
    assert np.flatnonzero(st["label"] != ref.label.astype(np.int32)).size <= 3
    ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    for _ in range(14):
        ref.step()
    ctx.step(14)
    st = ctx.download(psi=True, label=True)
    assert np.array_equal(st["psi"].view(np.uint32), ref.U.view(np.uint32))
    assert np.array_equal(st["label"], ref.label.astype(np.int32))
