"""The solver.py flavour end to end through the C ABI (Context / drop-in RealQMSolver)
against the oracle's restatement of RealQMSolver's schedule (oracle.SolverPyDriver).

Both use snapshot label semantics and FP64 per-domain norms.  The GPU normalisation sums
in a different order, so psi and energies agree to FP32 rounding, not bit for bit; labels
depend only on labels and atom positions in this flavour and agree exactly.
"""
import json
import os

import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def h2o_cfg():
    with open(os.path.join(GOLD, "solverpy_run_h2o_nn32.json")) as f:
        return json.load(f)["config"]


def glycine_like_cfg(NN=48, screen=12.0):
    rng = np.random.default_rng(5)
    N2 = NN // 2
    atoms = []
    for n in range(10):
        p = rng.uniform(N2 - 12, N2 + 12, 3)
        atoms.append({"i": float(np.round(p[0])), "j": float(np.round(p[1])), "k": float(np.round(p[2])),
                      "Z": float(rng.integers(1, 5)), "rc": float(rng.choice([0.0, 0.3, 0.4]))})
    return {"gridN": NN, "screen": screen, "atoms": atoms}


@pytest.mark.parametrize("cfg_fn,steps", [(h2o_cfg, 200), (glycine_like_cfg, 300)])
def test_context_matches_oracle_schedule(cfg_fn, steps):
    from realmolecule_b200 import Context, _lib as L
    cfg = cfg_fn()
    ref = orc.SolverPyDriver(cfg, kernels="oracle")
    ref.initialize()
    ctx = Context(cfg["gridN"], cfg["screen"], cfg["atoms"], flavor="solver.py")
    ctx.initialize()
    st0 = ctx.download(psi=True, label=True, P=True)
    assert np.array_equal(st0["label"], ref.label)
    np.testing.assert_allclose(st0["P"], ref.P, rtol=0, atol=2e-6 * np.abs(ref.P).max())
    ref.run(steps)
    ctx.step(steps)
    st = ctx.download(psi=True, label=True, P=True)
    assert np.array_equal(st["label"], ref.label)
    assert np.max(np.abs(st["psi"] - ref.U)) <= 1e-5 * np.abs(ref.U).max()
    e = ctx.energy()
    ref.energy()
    for k, v in ((L.E_T, ref.E_T), (L.E_EK, ref.E_eK), (L.E_EE, ref.E_ee), (L.E_KK, ref.E_KK)):
        assert abs(e[k] - v) <= 1e-5 * max(1.0, abs(v)), (k, e[k], v)


def test_graph_replay_equals_eager():
    """A period replayed from its CUDA graph gives the same bits as the same steps launched
    one by one (1 + 99 steps are eager, the next 100 come from the graph)."""
    from realmolecule_b200 import Context
    cfg = h2o_cfg()
    a = Context(cfg["gridN"], cfg["screen"], cfg["atoms"])
    b = Context(cfg["gridN"], cfg["screen"], cfg["atoms"])
    a.initialize(); b.initialize()
    a.step(100); a.step(100); a.step(100)     # graph captured, then replayed twice
    for _ in range(300):
        b.step(1)                              # never aligned to a full period: all eager
    sa, sb = a.download(psi=True, label=True), b.download(psi=True, label=True)
    assert np.array_equal(sa["label"], sb["label"])
    # FP64 atomics make the norms order-dependent at the last bit; psi agrees to rounding
    assert np.max(np.abs(sa["psi"] - sb["psi"])) <= 1e-6 * np.abs(sb["psi"]).max()


def test_dropin_solver_run_and_snapshots():
    from realmolecule_b200 import RealQMSolver
    cfg = dict(h2o_cfg())
    s = RealQMSolver(cfg)
    res = s.run(total_steps=200, report_interval=100)
    assert [r["step"] for r in res] == [100, 200]
    for key in ("E", "E_T", "E_eK", "E_ee", "E_KK", "E_bind", "ms_per_step", "elapsed_sec", "nucPos"):
        assert key in res[-1]
    ref = orc.SolverPyDriver(cfg, kernels="oracle")
    ref.initialize(); ref.run(200); ref.energy()
    assert abs(res[-1]["E"] - ref.E) < 1e-5 * abs(ref.E)
    assert s.U.shape == (33 ** 3,) and s.label.dtype == np.int32


def test_dropin_dynamics_moves_nuclei_like_reference_host_code():
    """Forces every 50 steps and the reference's damped Euler move: positions after the run
    agree with the oracle driver + the same host move to 1e-4 cells."""
    from realmolecule_b200 import RealQMSolver
    cfg = dict(h2o_cfg(), dynamics=True, force_interval=50, forceScale=50.0)
    s = RealQMSolver(cfg)
    s.run(total_steps=100, report_interval=100)
    ref = orc.SolverPyDriver(cfg, kernels="oracle")
    ref.initialize()
    vel = np.zeros((ref.nAtoms, 3), np.float32)
    for _ in range(2):
        ref.run(50)
        F = np.zeros(ref.nAtoms * 3)
        orc.O().sp_forces(ref.U, ref.atoms5, ref.nAtoms, ref.S, np.float32(ref.h), np.float32(ref.h2),
                          np.float32(ref.h3), F)
        F = F.reshape(-1, 3).astype(np.float32)
        F += nuclear_forces(ref)
        move(ref, F, vel, cfg)
    np.testing.assert_allclose(s.atom_pos, ref.atom_pos, atol=1e-4)


def nuclear_forces(ref):
    n = ref.nAtoms
    F = np.zeros((n, 3), np.float32)
    for a in range(n):
        for b in range(n):
            if a == b:
                continue
            d = (ref.atom_pos[a].astype(np.float64) - ref.atom_pos[b]) * ref.h
            r2 = float(d @ d) + ref.h2
            F[a] += (ref.Z_eff[a] * ref.Z_eff[b] / (r2 * np.sqrt(r2)) * d).astype(np.float32)
    return F


def move(ref, F, vel, cfg):
    mass = {1: 1836, 2: 16 * 1836, 3: 14 * 1836, 4: 12 * 1836}
    dt_nuc, damping, max_vel = 0.8, 0.98, 0.3
    for n in range(ref.nAtoms):
        z = int(ref.Z_eff[n])
        m = mass.get(z, 1836)
        for d in range(3):
            vel[n][d] += F[n][d] / m * dt_nuc * cfg["forceScale"]
            vel[n][d] *= damping
            vel[n][d] = np.clip(vel[n][d], -max_vel, max_vel)
            ref.atom_pos[n][d] += vel[n][d] * dt_nuc / ref.h
            ref.atom_pos[n][d] = np.clip(ref.atom_pos[n][d], 5, ref.NN - 5)
    a5 = ref.atoms5.reshape(-1, 5)
    a5[:, :3] = ref.atom_pos
    ref.atoms5 = np.ascontiguousarray(a5.reshape(-1))
    orc.O().sp_recompute_K(ref.K, ref.atoms5, ref.nAtoms, ref.S, np.float32(ref.h), np.float32(ref.h2))


def test_rejected_label_upload_leaves_the_state_unchanged():
    """Labels are checked on the device after the copy; a label outside [0, n_atoms) is reported
    (status RQ_EINVAL, index and value in the message) and the context keeps its state: the next
    steps give the same fields as on a twin context that never saw the upload."""
    from realmolecule_b200 import Context, _lib as L
    cfg = h2o_cfg()
    ctxs = [Context(cfg["gridN"], cfg["screen"], cfg["atoms"], flavor="solver.py") for _ in range(2)]
    for c in ctxs:
        c.initialize()
        c.step(30)
    st = ctxs[0].download(psi=True, label=True)
    bad = st["label"].copy()
    bad[1234] = len(cfg["atoms"]) + 5
    with pytest.raises(L.RqError) as e:
        ctxs[0].upload(label=bad)
    assert e.value.status == L.RQ_EINVAL and "index 1234" in str(e.value)
    assert np.array_equal(ctxs[0].download(psi=False, label=True)["label"], st["label"])
    ctxs[0].upload(label=st["label"])  # an accepted upload of the same labels changes nothing either
    for c in ctxs:
        c.step(130)  # crosses a label step
    a, b = (c.download(psi=True, label=True) for c in ctxs)
    assert np.array_equal(a["label"], b["label"])
    # psi: the FP64 domain sums of the normalisation are atomics in any order
    np.testing.assert_allclose(a["psi"], b["psi"], rtol=1e-6, atol=1e-9)
    for c in ctxs:
        c.close()
