"""CPU tests of the molecule.js page host (MoleculePage) with a stand-in context: the frame loop's
force cadence and convergence monitor, the nuclear forces, restraints and integrator of
moveNuclei, and the restarts.  The GPU side of the same host is in test_gpu_molecule_host.py."""
import math

import numpy as np
import pytest

from realmolecule_b200 import _lib as L
from realmolecule_b200.molecule_host import MoleculePage, nuc_mass


class FakeContext:
    """Prescribed energies and electronic forces; records the calls the host makes."""

    def __init__(self, n, E=(-1.0,), F=None):
        self.n, self.E, self.k = n, list(E), 0
        self.F = np.zeros((n, 3)) if F is None else np.asarray(F, float)
        self.steps, self.atoms, self.inits, self.splits = [], [], 0, []

    def step(self, n):
        self.steps.append(n)

    def energy(self):
        e = np.zeros(L.ENERGY_LEN)
        e[L.E_TOTAL] = self.E[min(self.k, len(self.E) - 1)]
        self.k += 1
        return e

    def forces(self, method):
        assert method == L.FORCE_GRADP
        return self.F.copy()

    def set_atoms(self, rows):
        self.atoms.append([(r["i"], r["j"], r["k"], r["Z"]) for r in rows])

    def initialize(self):
        self.inits += 1

    def extract(self, k=None):
        return np.zeros(1, np.float32)

    def set_locked_groups(self, groups):
        self.locked = groups

    def set_splits(self, splits):
        self.splits.append([dict(x) for x in splits])

    def restart(self):
        self.restarts = getattr(self, "restarts", 0) + 1

    def set_freeze_boundary(self, on):
        self.freeze = getattr(self, "freeze", []) + [bool(on)]


WATER = [{"i": 50, "j": 50, "k": 50, "Z": 2, "el": "O"}, {"i": 60, "j": 57, "k": 50, "Z": 1, "el": "H"},
         {"i": 40, "j": 57, "k": 50, "Z": 1, "el": "H"}]


def page(rows=WATER, F=None, E=(-1.0,), **kw):
    ctx = FakeContext(len(rows), E=E, F=F)
    return MoleculePage(rows, NN=100, screen=10.0, context=ctx, **kw), ctx


def test_forces_every_n_move_steps_and_page_defaults():
    p, ctx = page(steps_per_frame=5, dynamics=True)
    assert p.dt_nuc == 2.0 and p.substeps == 2 and p.max_vel == 0.3
    for _ in range(4):
        p.frame()
    assert ctx.steps == [5, 5, 5, 5]
    assert len(ctx.atoms) == 2  # moves after frames 2 and 4 (steps 10 and 20)


def test_site_repulsion_is_pairwise_and_shared_by_coincident_entries():
    rows = WATER + [{"i": 50, "j": 50, "k": 50, "Z": 1, "Z_nuc": 0.5}]
    p, _ = page(rows, dynamics=False)
    assert len(p.unique) == 3 and p.unique[0]["Z_eff"] == 2.5
    p.frame()
    p.frame()
    f = np.array(p.nuc_force_nuc)
    assert np.allclose(f[0], f[3])
    site_sum = f[0] + f[1] + f[2]
    assert np.allclose(site_sum, 0.0, atol=1e-12)


def test_frozen_hinge_clamp_damping_and_velocity_cap():
    F = np.array([[0.0, 0.0, 0.0], [5e3, 0.0, 0.0], [1e-3, 0.0, 0.0]])
    p, ctx = page(F=F, dynamics=True, frozen_atoms=[0], hinge_atoms=[2], no_nuc_repulsion=True, steps_per_frame=10)
    p.frame()
    assert p.pos[0] == [50.0, 50.0, 50.0]                       # frozen
    assert p.pos[2] == [40.0, 57.0, 50.0]                       # hinge: no force, no velocity
    assert p.nuc_vel[1][0] == pytest.approx(p.max_vel)          # capped
    assert p.pos[1][0] <= p.NN - 5                              # clamped to the box
    assert ctx.atoms[-1][1][0] == p.pos[1][0]                   # K rebuilt from the moved positions


def test_bond_and_angle_restraints_are_internal_forces():
    p, _ = page(dynamics=True, no_nuc_repulsion=True, bond_constraints=[[0, 1, 1.0, 2.0]],
                water_triplets=[[0, 1, 2]], steps_per_frame=10)
    p.frame()
    F = np.array(p.nuc_force)
    assert np.allclose(F.sum(axis=0), 0.0, atol=1e-12)
    r01 = (np.array(WATER[1]["i"]) - WATER[0]["i"]) * p.h
    assert F[1][0] < 0 < r01  # the stretched bond pulls H back towards O


def test_coincident_groups_move_together_and_rigid_groups_share_a_displacement():
    rows = WATER + [{"i": 60, "j": 57, "k": 50, "Z": 1}]
    F = np.array([[0, 0, 0], [1e-2, 0, 0], [0, 0, 0], [0, 2e-2, 0]], float)
    p, _ = page(rows, F=F, dynamics=True, no_nuc_repulsion=True, coincident_groups=[[1, 3]], steps_per_frame=10)
    p.frame()
    assert p.pos[3] == p.pos[1] and p.pos[1][1] > 57.0
    q, _ = page(F=F[:3], dynamics=True, no_nuc_repulsion=True, rigid_groups=[[1, 2]], steps_per_frame=10)
    q.frame()
    d1 = np.subtract(q.pos[1], [60, 57, 50])
    d2 = np.subtract(q.pos[2], [40, 57, 50])
    assert np.allclose(d1, d2) and d1[0] > 0
    assert q.nuc_vel[1][0] == pytest.approx((1e-2 / (2 * nuc_mass(1)) * q.dt_nuc) * q.damping
                                            * (1 + q.damping) if q.substeps == 2 else 0, rel=1e-12)


def test_thermostat_is_seeded_and_brownian_moves_without_velocity():
    a, _ = page(dynamics=True, langevin_kT=1e-3, langevin_gamma=1.0, seed=7, steps_per_frame=10)
    b, _ = page(dynamics=True, langevin_kT=1e-3, langevin_gamma=1.0, seed=7, steps_per_frame=10)
    a.frame(); b.frame()
    assert a.pos == b.pos and a.temperature() > 0
    c, _ = page(dynamics=True, brownian=True, langevin_kT=0.0, steps_per_frame=10,
                F=np.array([[0, 0, 0], [1e-2, 0, 0], [0, 0, 0]], float), no_nuc_repulsion=True)
    c.frame()
    assert c.pos[1][0] > 60 and c.nuc_vel[1] == [0.0, 0.0, 0.0]


def test_convergence_after_three_quiet_frames_and_auto_dynamics():
    E = [-1.0, -1.5] + [-1.6] * 20
    p, _ = page(E=E, convergence_threshold=1e-6, steps_per_frame=50)
    frames = 0
    while p.phase == 0 and frames < 30:
        p.frame()
        frames += 1
    assert p.converged_at is not None and p.converged_at > 200
    q, _ = page(steps_per_frame=50)
    for _ in range(200):
        q.frame()
    assert q.dynamics  # auto-enabled after 10000 steps


def test_restart_and_activate():
    p, ctx = page(dynamics=True, steps_per_frame=10)
    p.frame()
    p.restartWithPositions([[52, 50, 50], [62, 57, 50], [42, 57, 50]])
    assert ctx.inits == 1 and p.tStep == 0 and p.mol_pos[0] == [52.0, 50.0, 50.0]
    p.activateAtoms(2)
    assert ctx.inits == 2 and ctx.atoms[-1][2][3] == 0.0 and p.Z[:2] == [2.0, 1.0]
    assert p.pos[0] == [52.0, 50.0, 50.0]


def test_lobpcg_frames_count_ten_steps_and_skip_forces():
    """In LOBPCG mode a frame is one doLOBPCGStep (one rq_step) counted as LOBPCG_ITERS = 10 steps;
    the page computes no forces and moves no nuclei in it (molecule.js:3323-3740, :4614-4616)."""
    p, ctx = page(dynamics=True, n_move=10, lobpcg=1)
    for _ in range(3):
        p.frame()
    assert ctx.steps == [1, 1, 1]
    assert p.tStep == 30 and p.phase_steps == 30
    assert ctx.atoms == []  # no moveNuclei


def test_locked_groups_reach_the_context():
    p, ctx = page(locked_groups=[[0, 1], [2]])
    assert ctx.locked == [[0, 1], [2]]


def _sector(d, sp):
    """inSplitAtom's sector index (molecule.js:209-224) in double precision."""
    L = math.hypot(*sp["axis"])
    a = [x / L for x in sp["axis"]]
    dp = sum(d[c] * a[c] for c in range(3))
    p = [d[c] - dp * a[c] for c in range(3)]
    e1 = [a[1], -a[0], 0.0] if abs(a[2]) < 0.9 else [0.0, a[2], -a[1]]
    n = math.hypot(*e1)
    e1 = [x / n for x in e1]
    e2 = [a[1] * e1[2] - a[2] * e1[1], a[2] * e1[0] - a[0] * e1[2], a[0] * e1[1] - a[1] * e1[0]]
    th = math.atan2(sum(p[c] * e2[c] for c in range(3)), sum(p[c] * e1[c] for c in range(3))) - sp["rot"]
    th += 2 * math.pi if th < -math.pi else -2 * math.pi if th > math.pi else 0.0
    return int(math.floor((th + math.pi) / (2 * math.pi / 3))) % 3


def test_split_frames_follow_the_water_and_precede_each_rebuild():
    """updateSplitFrames (molecule.js:1840-1878): the O-site entries' sector frame puts the two O-H
    bonds in sectors 0 and 1 and the lone pair in sector 2, is pushed before the context is
    initialised and again before every rebuild after the nuclei move."""
    rows = [{"i": 50, "j": 50, "k": 50, "Z": 1}] * 3 + [{"i": 57, "j": 55, "k": 52, "Z": 1},
                                                         {"i": 43, "j": 56, "k": 49, "Z": 1}]
    p, ctx = page(rows=rows, splits=[{"type": "third", "idx": q} for q in range(3)],
                  split_groups=[{"o": [0, 1, 2], "h": [3, 4]}])
    assert len(ctx.splits) == 1 and ctx.atoms == []
    for move in range(2):
        sp = ctx.splits[-1]
        o = p.pos[0]
        d1, d2 = ([p.pos[e][c] - o[c] for c in range(3)] for e in (3, 4))
        lone = [-(d1[c] / math.hypot(*d1) + d2[c] / math.hypot(*d2)) for c in range(3)]
        assert [_sector(d, sp[0]) for d in (d1, d2, lone)] == [0, 1, 2]
        assert sp[0]["axis"] == sp[1]["axis"] == sp[2]["axis"] and sp[3]["type"] == 0
        p.pos[3] = [p.pos[3][0] + 1.5, p.pos[3][1] - 2.0, p.pos[3][2] + 0.7]  # the molecule turns
        p.restartWithPositions(p.pos)
        assert len(ctx.splits) == move + 2 and len(ctx.atoms) == move + 1


def test_hemi_split_group_uses_the_bisector():
    rows = [{"i": 50, "j": 50, "k": 50, "Z": 1}] * 2 + [{"i": 57, "j": 55, "k": 50, "Z": 1},
                                                         {"i": 43, "j": 55, "k": 50, "Z": 1}]
    p, ctx = page(rows=rows, splits=[{"type": "hemi", "idx": 0}, {"type": "hemi", "idx": 1}],
                  split_groups=[{"o": [0, 1], "h": [2, 3], "type": "hemi"}])
    ax = ctx.splits[-1][0]["axis"]
    assert abs(ax[0]) < 1e-12 and abs(ax[1] - 1.0) < 1e-12 and abs(ax[2]) < 1e-12


# three residues of two atoms each, Ca atoms 0, 2, 4 thirty cells (3 bohr) apart on the 0.1-bohr grid
# of page(): beyond the 3-angstrom steric minimum (56.7 cells) for the non-bonded pair 0-4
CHAIN = [{"i": 12 + 30 * r + d, "j": 50, "k": 50, "Z": 1} for r in range(3) for d in (0, 1)]
CMD = {"caIndices": [0, 2, 4], "groups": [[0, 1], [2, 3], [4, 5]], "mdDt": 10.0, "targetCaCa": 3.0}


def test_classical_md_translate_moves_residues_then_restarts():
    """USER_CLASSICAL_MD 'translate' (molecule.js:3929-4166): each residue moves by its summed force
    x forceScale x mdDt x 0.01, damped toward the pinned ends by (d+1)/3 at distance d < 2 from an
    end, capped at one cell; the electrons restart from scratch and the step counters reset."""
    F = np.zeros((6, 3))
    F[2:4, 1] = 0.2  # the middle residue is pulled along +j
    F[0:2, 2] = 0.1  # the first residue along +k
    p, ctx = page(rows=CHAIN, F=F, dynamics=True, n_move=5, steps_per_frame=5, no_nuc_repulsion=True,
                  classical_md=dict(CMD, mode="translate"))
    pos0 = [list(x) for x in p.pos]
    p.frame()
    assert getattr(ctx, "restarts", 0) == 1 and len(ctx.atoms) == 1
    assert p.tStep == 0 and p.phase_steps == 5
    dj = p.pos[2][1] - pos0[2][1]
    assert abs(dj - 0.4 * 10.0 * 0.01 * 2 / 3) < 1e-12  # middle residue: distance 1 from the ends
    assert abs((p.pos[0][2] - pos0[0][2]) - 0.2 * 10.0 * 0.01 / 3) < 1e-12  # first residue: damping 1/3
    assert p.pos[4] == pos0[4] and p.pos[5] == pos0[5]


def test_classical_md_shake_restores_the_ca_spacing():
    F = np.zeros((6, 3))
    F[4:6, 0] = 100.0  # the last residue pulled away: capped at one cell, then SHAKE pulls back
    p, ctx = page(rows=CHAIN, F=F, dynamics=True, n_move=5, steps_per_frame=5, no_nuc_repulsion=True,
                  classical_md=dict(CMD, mode="translate", shakeTolerance=0.01))
    p.frame()
    d = math.dist(p.pos[2], p.pos[4])
    assert 30.0 < d <= 30.0 * 1.01 + 1e-9  # stretched, and back within the tolerance


def test_classical_md_rigid_strands_turn_about_the_hinge():
    """The default mode (molecule.js:4167-4222): two strands turn about the hinge between residues
    hingeRes-1 and hingeRes by their torques, each angle capped at 0.02 rad."""
    rows = [{"i": 10 + 6 * r, "j": 20, "k": 20, "Z": 1} for r in range(4)]
    F = np.zeros((4, 3))
    F[0, 1] = 50.0   # strand 1 (residues 0, 1) pushed to +j: turns by the cap
    F[3, 1] = 1e-3   # strand 2: a small torque
    cmd = {"caIndices": [0, 1, 2, 3], "groups": [[0], [1], [2], [3]], "mdDt": 1.0}
    p, ctx = page(rows=rows, F=F, dynamics=True, n_move=5, steps_per_frame=5, no_nuc_repulsion=True,
                  classical_md=cmd)
    hinge = (19.0, 20.0)
    pos0 = [list(x) for x in p.pos]
    p.frame()
    for a in range(4):  # rotations keep the distance to the hinge
        r0 = math.hypot(pos0[a][0] - hinge[0], pos0[a][1] - hinge[1])
        assert abs(math.hypot(p.pos[a][0] - hinge[0], p.pos[a][1] - hinge[1]) - r0) < 1e-9
    th1 = math.atan2(p.pos[0][1] - hinge[1], p.pos[0][0] - hinge[0]) - math.pi
    assert abs(abs(th1) - 0.02) < 1e-12
    th2 = math.atan2(p.pos[3][1] - hinge[1], p.pos[3][0] - hinge[0])
    assert 0 < th2 < 0.02
    assert getattr(ctx, "restarts", 0) == 1


def test_init_zeff_and_rcut_follow_fill_atom_buf():
    """fillAtomBuf (molecule.js:1886-1891): the per-atom lists win, a 0 entry falls back to Z (and
    1e6 for the radius); without a list the page-wide INIT_ZEFF / INIT_RCUT, else Z / 1e6."""
    p, ctx = page(init_zeff=1.7, init_rcut=3.0)
    p.restartWithPositions(p.pos)
    assert [(r[3]) for r in ctx.atoms[-1]] == [2, 1, 1]
    assert [p._init_params(e) for e in range(3)] == [(1.7, 3.0)] * 3
    p, ctx = page(init_zeff=1.7, user_init_zeff=[3.1, 0, 0.9], user_init_rcut=[0, 2.5])
    assert [p._init_params(e) for e in range(3)] == [(3.1, 1e6), (1.0, 2.5), (0.9, 1e6)]
    rows = p._ctx_rows()
    assert rows[0]["initZeff"] == 3.1 and rows[1]["initRcut"] == 2.5
    p, ctx = page()
    assert "initZeff" not in p._ctx_rows()[0]  # nothing set: the rows carry no override


def test_freeze_boundary_until_the_unlock_step():
    """FREEZE_BOUNDARY with UNLOCK_AT_STEP (molecule.js:4621-4624): frozen from the start, released
    once phaseSteps reaches the unlock step."""
    p, ctx = page(steps_per_frame=5, freeze_boundary=True, unlock_at_step=12)
    assert ctx.freeze == [True]
    p.frame()
    p.frame()
    assert ctx.freeze == [True] and p.freeze_boundary
    p.frame()  # phase_steps 15 >= 12
    assert ctx.freeze == [True, False] and not p.freeze_boundary
    p.frame()
    assert ctx.freeze == [True, False]


def test_from_page_reads_the_page_globals():
    """from_page builds rows and options from a page's window globals as molecule.js reads them
    (molecule.js:4-152): k defaults to round(NN/2), only the first NELEC entries count, `||` options
    take their defaults when falsy, temperatures become kT = T / 315775."""
    g = {"USER_NN": 120, "USER_SCREEN": 12.0,
         "USER_ATOMS": [{"i": 60, "j": 60, "el": "O"}, {"i": 66, "j": 64, "k": 58, "el": "H"},
                        {"i": 54, "j": 64, "el": "H"}, {"i": 10, "j": 10, "el": ""}],
         "USER_Z": [6, 1, 1, 0], "USER_RC": [0.4, 0, 0, 0], "USER_DT_NUC": 0, "USER_TEMPERATURE_K": 300,
         "USER_LOCKED_GROUPS": [[0, 1]], "USER_CURV_REG": 0, "USER_DV": 0.1, "FREEZE_BOUNDARY": True,
         "UNLOCK_AT_STEP": 500, "INIT_ZEFF": 1.7}
    ctx = FakeContext(3)
    p = MoleculePage.from_page(g, context=ctx)
    assert p.n == 3 and p.NN == 120 and p.screen == 12.0
    assert [r["k"] for r in p.rows] == [60, 58, 60] and [r["Z"] for r in p.rows] == [6, 1, 1]
    assert p.rows[0]["rc"] == 0.4 and p.rows[1]["Z_nuc"] == 1
    assert abs(p.langevin_kT - 300 / 315775.0) < 1e-15
    assert p.dt_nuc == 2.0  # USER_DT_NUC = 0 falls back to the default for <= 5 entries
    assert ctx.locked == [[0, 1]] and ctx.freeze == [True] and p.unlock_at_step == 500
    assert p._init_params(0) == (1.7, 1e6)
