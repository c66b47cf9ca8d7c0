"""The host side of a molecule.js page around the GPU step (molecule.js flavour of librq).

molecule.js runs its frames on the GPU and everything else in the page's JavaScript: the frame
loop and its convergence monitor (draw, molecule.js:4584-4671), the nuclear forces (the GPU's
Hartree gradient plus the softened repulsion of the unique nuclei, :3205-3259), the nuclear
integrator with its restraints and thermostats (moveNuclei, :3742-4583), the warm K rebuild
after a move, and the restarts (restartWithPositions / activateAtoms, :2127-2195).
``MoleculePage`` is that host over a ``Context(flavor="molecule.js")``; option names follow the
page's ``window.USER_*`` globals.  Positions are grid coordinates (i, j, k).

Kept from moveNuclei: user external forces, hinge atoms, bond-length and H-O-H angle
restraints, coincident groups, rigid groups, frozen atoms, the shear body force, overdamped
Brownian motion, the Andersen thermostat (a seeded generator stands in for Math.random) and the
coarse-grained classical-MD backbone with its SASA pressure and full restart (USER_CLASSICAL_MD,
USER_SASA).  Page options of the GPU frame: locked groups, shell splits and their water frames,
FREEZE_BOUNDARY / UNLOCK_AT_STEP, INIT_ZEFF / INIT_RCUT, and the LOBPCG solver (lobpcg=1).
Not kept: the fold-force diagnostics (USER_FOLD_ATOMS), which only log.
"""
from __future__ import annotations

import math
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib as L
from .context import Context

_MASS = {1: 1, 2: 16, 3: 14, 4: 12}


def nuc_mass(z: float) -> float:
    """molecule.js:152 -- mass by valence charge (H, O, N, C pseudo-atoms) in electron masses."""
    return _MASS.get(z, 1) * 1836


LOBPCG_ITERS = 10  # molecule.js:1752, iterations per domain in one LOBPCG frame


class MoleculePage:
    def __init__(self, atoms: Sequence[dict], NN: int = 100, screen: float = 10.0, steps_per_frame: Optional[int] = None,
                 total_steps: int = 20000, n_move: int = 10, dynamics: bool = False, dt_nuc: Optional[float] = None,
                 nuc_substeps: Optional[int] = None, damping: float = 0.98, force_scale: float = 1.0,
                 langevin_kT: float = 0.0, langevin_gamma: float = 0.01, no_nuc_repulsion: bool = False,
                 no_auto_dynamics: bool = False, convergence_threshold: Optional[float] = None,
                 external_force=None, hinge_atoms=(), frozen_atoms=(), bond_constraints=(), water_triplets=(),
                 hoh_eq: float = 104.5, bend_k: float = 1.5, coincident_groups=(), rigid_groups=None,
                 shear_rate: float = 0.0, brownian: bool = False, brownian_gamma: float = 1.0,
                 thermal_kick: Optional[float] = None, seed: int = 0, locked_groups=(), splits=(), split_groups=(),
                 classical_md=None, sasa=None, init_zeff=None, init_rcut=None, user_init_zeff=None,
                 user_init_rcut=None, freeze_boundary=False, unlock_at_step=None, init_pos=None, context=None,
                 **ctx_opts):
        self.rows = [dict(a) for a in atoms]
        n = self.n = len(self.rows)
        # USER_INIT_POS (molecule.js:1909-1921): per entry (i, j) of its trial psi, or None
        self.init_pos = [None if p is None else (float(p[0]), float(p[1])) for p in (init_pos or [])]
        self.NN, self.screen = int(NN), float(screen)
        self.h = self.screen / self.NN
        self.Z_orig = [float(a.get("Z", 0.0)) for a in self.rows]
        self.Z_nuc = [float(a["Z_nuc"]) if a.get("Z_nuc") is not None else float(a.get("Z", 0.0)) for a in self.rows]
        self.Z = list(self.Z_orig)
        # the trial psi's exponent and cut-off radius (fillAtomBuf, molecule.js:1886-1891): per atom
        # USER_INIT_ZEFF / USER_INIT_RCUT, else the page-wide INIT_ZEFF / INIT_RCUT, else Z / 1e6
        self.init_zeff, self.init_rcut = init_zeff, init_rcut
        self.user_init_zeff, self.user_init_rcut = user_init_zeff, user_init_rcut
        self.mol_pos = [[float(a["i"]), float(a["j"]), float(a.get("k", self.NN // 2))] for a in self.rows]
        self.pos = [list(p) for p in self.mol_pos]
        # molecule.js:106, :116-121 -- defaults by the number of entries
        self.spf = steps_per_frame or (50 if n <= 30 else 5 if n <= 100 else 2)
        self.total_steps, self.n_move = int(total_steps), int(n_move)
        self.dt_nuc = dt_nuc or (2.0 if n <= 5 else 0.2 if n > 200 else 0.8)
        self.substeps = nuc_substeps or (2 if n <= 5 else 1)
        self.damping, self.force_scale = float(damping), float(force_scale)
        self.max_vel = 0.3 if n <= 5 else 0.03 if n > 200 else 0.1
        self.langevin_kT, self.langevin_gamma = float(langevin_kT), float(langevin_gamma)
        self.add_nuc_repulsion = not no_nuc_repulsion
        self.no_auto_dynamics = bool(no_auto_dynamics)
        self.convergence_threshold = convergence_threshold
        self.dynamics = bool(dynamics)
        self.external_force = external_force
        self.hinge_atoms, self.frozen_atoms = list(hinge_atoms), set(frozen_atoms)
        self.bond_constraints, self.water_triplets = list(bond_constraints), list(water_triplets)
        self.hoh_eq, self.bend_k = float(hoh_eq), float(bend_k)
        self.coincident_groups, self.rigid_groups = list(coincident_groups), rigid_groups
        self.shear_rate, self.brownian, self.brownian_gamma = float(shear_rate), bool(brownian), float(brownian_gamma)
        self.thermal_kick = thermal_kick
        # USER_CLASSICAL_MD / USER_SASA (molecule.js:3856-4291): the coarse-grained backbone mode
        self.classical_md, self.sasa = classical_md, sasa
        self.compact_rg = None
        self.rng = np.random.default_rng(seed)
        self._unique_nuclei()
        # `context`: an object with the Context methods used here (tests drive the host logic with one)
        self.ctx = context if context is not None else Context(self.NN, self.screen, self._ctx_rows(),
                                                               flavor="molecule.js", steps_per_frame=self.spf,
                                                               **ctx_opts)
        # useLOBPCG (molecule.js:1751): a frame is one doLOBPCGStep, counted as LOBPCG_ITERS steps
        self.lobpcg = bool(ctx_opts.get("lobpcg"))
        # USER_LOCKED_GROUPS (molecule.js:490-503)
        self.locked_groups = [list(g) for g in locked_groups]
        if self.locked_groups:
            self.ctx.set_locked_groups(self.locked_groups)
        # USER_SPLIT_TYPE / _IDX / _AXIS / _ROT per entry (molecule.js:27-32) and USER_SPLIT_GROUPS,
        # whose sector frames follow the water molecules (updateSplitFrames, :1840-1878)
        sp = list(splits) + [None] * (n - len(splits))
        self.split_type = [(s or {}).get("type", 0) for s in sp]
        self.split_idx = [int((s or {}).get("idx", 0)) for s in sp]
        self.split_axis = [list((s or {}).get("axis") or (0.0, 0.0, 1.0)) for s in sp]
        self.split_rot = [float((s or {}).get("rot", 0.0)) for s in sp]
        self.split_groups = [dict(g) for g in split_groups]
        self._push_splits()
        # window.FREEZE_BOUNDARY / UNLOCK_AT_STEP (molecule.js:3095, :3643, :4621-4624)
        self.freeze_boundary, self.unlock_at_step = bool(freeze_boundary), unlock_at_step
        if self.freeze_boundary:
            self.ctx.set_freeze_boundary(True)
        self._reset_counters()
        self.nuc_vel = [[0.0, 0.0, 0.0] for _ in range(n)]
        self.nuc_force = [[0.0, 0.0, 0.0] for _ in range(n)]
        self.nuc_force_total = [[0.0, 0.0, 0.0] for _ in range(n)]
        self.nuc_steps = 0

    @classmethod
    def from_page(cls, g: Dict, context=None) -> "MoleculePage":
        """Build from a dict of a molecule.js page's window globals (molecule.js:4-152 and the
        options read later): USER_ATOMS (i, j and optionally k, else round(NN/2)) with USER_Z,
        USER_Z_NUC and USER_RC per entry -- the first NELEC entries, those with Z > 0 or Z_nuc > 0
        counted as the page counts them -- and every page option MoleculePage keeps.  Options the
        page reads with `||` take their defaults when falsy; USER_BEND_K and USER_CURV_REG keep an
        explicit 0 (a curvature term of 0 is off)."""
        def js(key):  # `window.KEY || default`: falsy means unset
            v = g.get(key)
            return v if v else None

        NN = js("USER_NN") or 200
        z = list(js("USER_Z") or [2, 3, 1, 0, 0])
        zn = list(js("USER_Z_NUC") or z)
        rc = list(js("USER_RC") or [])
        atoms = list(js("USER_ATOMS") or [{"i": 80, "j": 120}, {"i": 100, "j": 77}, {"i": 120, "j": 120},
                                           {"i": 100, "j": 100}, {"i": 100, "j": 100}])
        at = lambda a, n, d=0.0: a[n] if n < len(a) and a[n] else d  # noqa: E731
        nelec = sum(1 for n in range(len(atoms)) if at(z, n) > 0 or at(zn, n) > 0) or 3
        rows = []
        for n in range(nelec):
            a = atoms[n] if n < len(atoms) else {"i": round(NN / 2), "j": round(NN / 2)}
            rows.append({"i": a["i"], "j": a["j"], "k": a.get("k", round(NN / 2)), "Z": at(z, n),
                         "Z_nuc": zn[n] if n < len(zn) else at(z, n), "rc": at(rc, n), "el": a.get("el", "")})
        kw = {"NN": NN, "screen": js("USER_SCREEN") or 10.0}
        for key, name in (("USER_STEPS_PER_FRAME", "steps_per_frame"), ("USER_STEPS", "total_steps"),
                          ("USER_N_MOVE", "n_move"), ("USER_DYNAMICS", "dynamics"), ("USER_DT_NUC", "dt_nuc"),
                          ("USER_NUC_SUBSTEPS", "nuc_substeps"), ("USER_DAMPING", "damping"),
                          ("USER_FORCE_SCALE", "force_scale"), ("USER_LANGEVIN_GAMMA", "langevin_gamma"),
                          ("NO_NUC_REPULSION", "no_nuc_repulsion"), ("NO_AUTO_DYNAMICS", "no_auto_dynamics"),
                          ("CONVERGENCE_THRESHOLD", "convergence_threshold"),
                          ("USER_EXTERNAL_FORCE", "external_force"), ("USER_HINGE_ATOMS", "hinge_atoms"),
                          ("USER_FROZEN_ATOMS", "frozen_atoms"), ("USER_BOND_CONSTRAINTS", "bond_constraints"),
                          ("USER_WATER_TRIPLETS", "water_triplets"), ("USER_HOH_EQ", "hoh_eq"),
                          ("USER_COINCIDENT_GROUPS", "coincident_groups"), ("USER_RIGID_GROUPS", "rigid_groups"),
                          ("USER_SHEAR_RATE", "shear_rate"), ("USER_BROWNIAN", "brownian"),
                          ("USER_BROWNIAN_GAMMA", "brownian_gamma"), ("USER_THERMAL_KICK", "thermal_kick"),
                          ("USER_LOCKED_GROUPS", "locked_groups"), ("USER_SPLIT_GROUPS", "split_groups"),
                          ("USER_CLASSICAL_MD", "classical_md"), ("USER_SASA", "sasa"), ("INIT_ZEFF", "init_zeff"),
                          ("INIT_RCUT", "init_rcut"), ("USER_INIT_ZEFF", "user_init_zeff"), ("USER_INIT_POS", "init_pos"),
                          ("USER_INIT_RCUT", "user_init_rcut"), ("FREEZE_BOUNDARY", "freeze_boundary"),
                          ("UNLOCK_AT_STEP", "unlock_at_step"),
                          # context options of the GPU frame
                          ("USER_DV", "dv"), ("USER_JACOBI_PER_STEP", "jacobi_per_step"),
                          ("USER_POISSON_INTERVAL", "vcycle_interval")):
            if js(key) is not None:
                kw[name] = js(key)
        if js("USER_TEMPERATURE_K"):  # kT = T / 315775 Ha (molecule.js:123-128)
            kw["langevin_kT"] = g["USER_TEMPERATURE_K"] / 315775.0
        if g.get("USER_BEND_K") is not None:
            kw["bend_k"] = g["USER_BEND_K"]
        if g.get("USER_CURV_REG") is not None:  # 0 switches the curvature term off
            kw["curv_reg"] = g["USER_CURV_REG"] if g["USER_CURV_REG"] else -1.0
        st = list(g.get("USER_SPLIT_TYPE") or [])
        if st:
            si, sa, sr = (list(g.get(k) or []) for k in ("USER_SPLIT_IDX", "USER_SPLIT_AXIS", "USER_SPLIT_ROT"))
            kw["splits"] = [{"type": at(st, n, 0), "idx": at(si, n, 0), "axis": at(sa, n, [0, 0, 1]),
                             "rot": at(sr, n, 0.0)} for n in range(nelec)]
        kw["sic"] = 1  # the page's own Pother path (direct Poisson for <= 5 domains, else the correction)
        return cls(rows, context=context, **kw)

    # ---- set-up ---------------------------------------------------------------------------------
    def _unique_nuclei(self):
        """molecule.js:50-66 -- entries at one site share one nucleus of charge sum(Z_nuc || Z)."""
        sites: Dict[tuple, dict] = {}
        for e, a in enumerate(self.rows):
            if self.Z_orig[e] == 0 and self.Z_nuc[e] == 0:
                continue
            key = (a["i"], a["j"], a.get("k", self.NN // 2))
            q = self.Z_nuc[e] or self.Z_orig[e]
            if key in sites:
                sites[key]["Z_eff"] += q
                sites[key]["elec"].append(e)
            else:
                sites[key] = {"Z_eff": q, "elec": [e]}
        self.unique = list(sites.values())

    def _init_params(self, e):
        """fillAtomBuf's initZeff / initRcut of entry e (molecule.js:1886-1891)."""
        zl, rl = self.user_init_zeff, self.user_init_rcut
        zeff = ((zl[e] if e < len(zl) else 0) or self.Z[e]) if zl else (self.init_zeff or self.Z[e])
        rcut = ((rl[e] if e < len(rl) else 0) or 1e6) if rl else (self.init_rcut or 1e6)
        return float(zeff), float(rcut)

    def _ctx_rows(self):
        rows = []
        for e, a in enumerate(self.rows):
            r = dict(a)
            r["i"], r["j"], r["k"] = self.pos[e]
            r["Z"], r["Z_nuc"] = self.Z[e], self.Z_nuc[e] if self.Z[e] or self.Z_nuc[e] else 0.0
            if self.init_zeff or self.init_rcut or self.user_init_zeff or self.user_init_rcut:
                r["initZeff"], r["initRcut"] = self._init_params(e)
            rows.append(r)
        return rows

    # ---- the coarse-grained classical-MD backbone (molecule.js:3856-4291) -------------------------
    def _moves(self, a) -> bool:
        return a < self.n and self.Z[a] != 0

    def _shift(self, group, d, sign=1.0):
        for a in group:
            if self._moves(a):
                for c in range(3):
                    self.pos[a][c] += sign * d[c]

    def _classical_md(self, F):
        """USER_CLASSICAL_MD: residues (groups, Ca atoms caIndices) move as rigid bodies under their
        summed nuclear forces -- plus the SASA pressure toward the Ca centroid (USER_SASA) -- either
        by per-residue translation ('translate': end damping, contact-driven damping of the quantum
        forces, a helical radial bias, SHAKE on Ca-Ca distances, Ca-Ca steric repulsion, H-bond and
        contact biases) or as two rigid strands turning about the hinge (default); positions are
        clamped to [5, NN-5], and the electrons restart from scratch (rq_restart, :4236-4286) with
        the step counters reset."""
        cmd, pos, h, NN = self.classical_md, self.pos, self.h, self.NN
        ca, groups = list(cmd["caIndices"]), [list(g) for g in cmd["groups"]]
        nres, md_dt, fscale = len(ca), float(cmd["mdDt"]), self.force_scale
        res = [[0.0, 0.0, 0.0] for _ in range(nres)]
        for g in range(nres):  # 1. summed quantum forces per residue
            for a in groups[g]:
                if self._moves(a):
                    for c in range(3):
                        res[g][c] += F[a][c]
        if self.sasa:  # SASA: exposed residues pushed toward the Ca centroid (:3885-3927)
            probe = self.sasa.get("probeRadius") or 15.0
            gamma = self.sasa.get("gamma") or 0.5
            max_nb = self.sasa.get("maxNeighbors") or 6
            cen = [sum(pos[ca[g]][c] for g in range(nres)) / nres for c in range(3)]
            for g in range(nres):
                p = pos[ca[g]]
                nb = sum(1 for q in range(nres) if q != g and
                         sum((pos[ca[q]][c] - p[c]) ** 2 for c in range(3)) < probe * probe)
                exposure = max(0.0, 1 - nb / max_nb)
                if exposure > 0:
                    d = [cen[c] - p[c] for c in range(3)]
                    dist = math.sqrt(sum(x * x for x in d)) + 0.01
                    for c in range(3):
                        res[g][c] += gamma * exposure * d[c] / dist
        if cmd.get("mode") == "translate":
            self._md_translate(cmd, ca, groups, res, md_dt, fscale)
        else:
            self._md_rigid_strands(cmd, ca, groups, res, md_dt, fscale)
        for a in range(self.n):  # boundary clamp (:4224-4230)
            if self.Z[a] != 0:
                pos[a] = [max(5.0, min(NN - 5.0, x)) for x in pos[a]]
        self.nuc_steps += 1
        self._push_splits()  # fillAtomBuf (:4237)
        self.ctx.set_atoms(self._ctx_rows())
        self.ctx.restart()
        self.tStep = 0
        self.phase_steps = 0

    def _md_translate(self, cmd, ca, groups, res, md_dt, fscale):
        pos, h, nres = self.pos, self.h, len(ca)
        max_disp = 1.0
        pin_n = 0 if cmd.get("pinEnds") is False else 2
        cb = cmd.get("contactBias")
        q_damp = 1.0
        if cb:  # quantum forces damped while a contact is far from its target (:3937-3955)
            excess_max = 0.0
            for pr in list(cb.get("hbonds") or []) + list(cb.get("contacts") or []):
                d = math.sqrt(sum((pos[pr["b"]][c] - pos[pr["a"]][c]) ** 2 for c in range(3))) * h
                excess_max = max(excess_max, (d - pr["target"]) / pr["target"])
            q_damp = 0.0 if excess_max > 1.0 else 0.1 if excess_max > 0.5 else 0.5 if excess_max > 0.2 else 1.0

        def capped(f, damp):
            d = [f[c] * fscale * md_dt * 0.01 * damp for c in range(3)]
            mag = math.sqrt(sum(x * x for x in d))
            return [x * max_disp / mag for x in d] if mag > max_disp else d

        for g in range(nres):
            end_damp = 1.0
            if pin_n > 0:
                dfe = min(g, nres - 1 - g)
                if dfe < pin_n:
                    end_damp = (dfe + 1) / (pin_n + 1)
            self._shift(groups[g], capped(res[g], end_damp * q_damp))
        if len(groups) > nres:  # the C-terminal group follows the last residue
            self._shift(groups[nres], capped(res[nres - 1], 1.0))
        hb = cmd.get("helicalBias")
        if hb:  # radial nudge toward the ideal helix radius (:3988-4034)
            c0, cl = pos[ca[0]], pos[ca[nres - 1]]
            ax = [cl[c] - c0[c] for c in range(3)]
            al = math.sqrt(sum(x * x for x in ax)) + 1e-10
            ax = [x / al for x in ax]
            cen = [sum(pos[ca[g]][c] for g in range(nres)) / nres for c in range(3)]
            r_ideal = (hb.get("idealRadius") or 4.35) / h
            strength = hb.get("strength") or 0.02
            for g in range(1, nres):
                r = [pos[ca[g]][c] - cen[c] for c in range(3)]
                axial = sum(r[c] * ax[c] for c in range(3))
                p = [r[c] - axial * ax[c] for c in range(3)]
                pl = math.sqrt(sum(x * x for x in p)) + 1e-10
                radial = (r_ideal - pl) * strength
                self._shift(groups[g], [p[c] / pl * radial for c in range(3)])
        target = (cmd.get("targetCaCa") or 7.18) / h  # SHAKE on Ca-Ca distances (:4037-4064)
        tol = cmd.get("shakeTolerance") or 0.15
        lo, hi = target * (1 - tol), target * (1 + tol)
        for _ in range(5):
            for g in range(nres - 1):
                a1, a2 = ca[g], ca[g + 1]
                d = [pos[a2][c] - pos[a1][c] for c in range(3)]
                dist = math.sqrt(sum(x * x for x in d))
                if dist < lo or dist > hi:
                    corr = ((lo if dist < lo else hi) - dist) / (2 * dist + 1e-10)
                    cv = [x * corr for x in d]
                    self._shift(groups[g], cv, -1.0)
                    self._shift(groups[g + 1], cv)
        min_nb = 3.0 * 1.8897 / h  # Ca-Ca steric repulsion beyond bonded neighbours (:4066-4094)
        for g1 in range(nres):
            for g2 in range(g1 + 2, nres):
                d = [pos[ca[g2]][c] - pos[ca[g1]][c] for c in range(3)]
                dist = math.sqrt(sum(x * x for x in d)) + 1e-10
                if dist < min_nb:
                    push = 0.5 * (min_nb - dist) / dist
                    pv = [x * push * 0.5 for x in d]
                    self._shift(groups[g1], pv, -1.0)
                    self._shift(groups[g2], pv)
        if cb:  # H-bond and contact biases (:4096-4161)
            owner = {}
            for g, grp in enumerate(groups):
                for a in grp:
                    owner[a] = g  # the last group holding an atom, as the page's search keeps

            def pair_bias(a, b, target_au, strength):
                d = [pos[b][c] - pos[a][c] for c in range(3)]
                dg = math.sqrt(sum(x * x for x in d)) + 1e-10
                if dg * h <= target_au:
                    return
                nudge = strength * (dg * h - target_au) / (dg * h)
                nv = [x / dg * nudge * 0.5 for x in d]
                if a in owner:
                    self._shift(groups[owner[a]], nv)
                if b in owner:
                    self._shift(groups[owner[b]], nv, -1.0)

            for pr in cb.get("hbonds") or []:
                pair_bias(pr["a"], pr["b"], pr["target"], cb.get("hbondStrength") or 0.5)
            for pr in cb.get("contacts") or []:
                pair_bias(pr["a"], pr["b"], pr["target"], cb.get("contactStrength") or 1.0)
            cm = [sum(pos[ca[g]][c] for g in range(nres)) / nres for c in range(3)]
            rg2 = sum(sum((pos[ca[g]][c] - cm[c]) ** 2 for c in range(3)) for g in range(nres))
            self.compact_rg = math.sqrt(rg2 / nres) * h

    def _md_rigid_strands(self, cmd, ca, groups, res, md_dt, fscale):
        pos, nres = self.pos, len(ca)
        hinge = cmd.get("hingeRes") or nres // 2
        hx = (pos[ca[hinge - 1]][0] + pos[ca[hinge]][0]) / 2
        hy = (pos[ca[hinge - 1]][1] + pos[ca[hinge]][1]) / 2
        t1 = sum((pos[ca[g]][0] - hx) * res[g][1] - (pos[ca[g]][1] - hy) * res[g][0] for g in range(hinge))
        t2 = sum((pos[ca[g]][0] - hx) * res[g][1] - (pos[ca[g]][1] - hy) * res[g][0] for g in range(hinge, nres))
        max_angle = 0.02
        th1 = max(-max_angle, min(max_angle, t1 * fscale * md_dt * 0.0001))
        th2 = max(-max_angle, min(max_angle, t2 * fscale * md_dt * 0.0001))

        def turn(group, th):
            cs, sn = math.cos(th), math.sin(th)
            for a in group:
                if self._moves(a):
                    rx, ry = pos[a][0] - hx, pos[a][1] - hy
                    pos[a][0], pos[a][1] = hx + rx * cs - ry * sn, hy + rx * sn + ry * cs

        for g in range(hinge):
            turn(groups[g], th1)
        for g in range(hinge, nres):
            turn(groups[g], th2)
        if len(groups) > nres:
            turn(groups[nres], th2)

    def _update_split_frames(self):
        """updateSplitFrames (molecule.js:1840-1878): for each water of USER_SPLIT_GROUPS ({o: the O-site
        entries, h: the two H entries, type}), the sector axis is the molecular-plane normal and the
        offset puts the two O-H bonds in sectors 0 and 1 and the lone pair in sector 2; a 'hemi'
        group splits along the H-H bisector instead."""
        for g in self.split_groups:
            o, h1, h2 = self.pos[g["o"][0]], self.pos[g["h"][0]], self.pos[g["h"][1]]
            u1 = [h1[c] - o[c] for c in range(3)]
            u2 = [h2[c] - o[c] for c in range(3)]
            n1, n2 = math.hypot(*u1) or 1.0, math.hypot(*u2) or 1.0
            u1 = [x / n1 for x in u1]
            u2 = [x / n2 for x in u2]
            a = [u1[1] * u2[2] - u1[2] * u2[1], u1[2] * u2[0] - u1[0] * u2[2], u1[0] * u2[1] - u1[1] * u2[0]]
            na = math.hypot(*a)
            if na < 1e-4:  # collinear: any normal
                a, na = [0.0, 0.0, 1.0], 1.0
            a = [x / na for x in a]
            b = [u1[c] + u2[c] for c in range(3)]
            nb = math.hypot(*b) or 1.0
            b = [x / nb for x in b]
            if g.get("type") == "hemi":
                for e in g["o"]:
                    self.split_axis[e], self.split_rot[e] = list(b), 0.0
                continue
            e1 = [a[1], -a[0], 0.0] if abs(a[2]) < 0.9 else [0.0, a[2], -a[1]]
            ne1 = math.hypot(*e1) or 1.0
            e1 = [x / ne1 for x in e1]
            e2 = [a[1] * e1[2] - a[2] * e1[1], a[2] * e1[0] - a[0] * e1[2], a[0] * e1[1] - a[1] * e1[0]]
            rot = math.atan2(sum(b[c] * e2[c] for c in range(3)), sum(b[c] * e1[c] for c in range(3))) + math.pi / 3
            for e in g["o"]:
                self.split_axis[e], self.split_rot[e] = list(a), rot

    def _push_splits(self):
        if not self.split_groups and not any(t not in (0, 1, "sphere", None) for t in self.split_type):
            return
        self._update_split_frames()
        self.ctx.set_splits([{"type": t, "idx": i, "axis": ax, "rot": r}
                             for t, i, ax, r in zip(self.split_type, self.split_idx, self.split_axis, self.split_rot)])

    def _upload_atoms(self):
        """fillAtomBuf + the device rebuild (molecule.js:1879-1903, :4563-4582): the split frames are
        recomputed from the new positions before the rebuild labels cells with them."""
        self._push_splits()
        self.ctx.set_atoms(self._ctx_rows())

    def _reset_counters(self):
        self.tStep = self.phase_steps = self.frame_count = 0
        self.E_min = math.inf
        self.phase = 0
        self._prevE = None
        self._conv_count = 0
        self.converged_at = None

    def initialize(self):
        """uploadInitialData on the device (with USER_INIT_POS, molecule.js:1905-1981, when given)."""
        if self.init_pos:
            self.ctx.set_init_positions(self.init_pos)
        self.ctx.initialize()
        self._reset_counters()

    # ---- the frame loop -------------------------------------------------------------------------
    def frame(self) -> Dict:
        """One draw() tick (molecule.js:4612-4671): a frame of steps, the energies, the nuclear forces
        when a force step fell in the frame (every N_MOVE steps, :2997-3004) and, with dynamics on,
        moveNuclei; then the auto-dynamics, convergence and end-of-run checks."""
        if self.phase != 0:
            return self.energies()
        t0 = self.tStep
        # doLOBPCGStep computes no forces and moves no nuclei (molecule.js:3323-3740, :4614-4616)
        nsteps = LOBPCG_ITERS if self.lobpcg else self.spf
        self.ctx.step(1 if self.lobpcg else self.spf)
        self.tStep += nsteps
        e = self.ctx.energy()
        self.E, self.E_T, self.E_eK, self.E_ee, self.E_KK = (float(e[L.E_TOTAL]), float(e[L.E_T]), float(e[L.E_EK]),
                                                             float(e[L.E_EE]), float(e[L.E_KK]))
        # forces are read on the frame's final state: the reference's last force step of the frame is
        # its final step whenever frames end on multiples of N_MOVE (every default frame length)
        if not self.lobpcg and any((t0 + s + 1) % self.n_move == 0 for s in range(self.spf)):
            self._forces()
            if self.dynamics:
                self.move_nuclei()
        self.phase_steps += nsteps
        if self.freeze_boundary and self.unlock_at_step and self.phase_steps >= self.unlock_at_step:
            self.freeze_boundary = False  # the boundaries move from the next frame on (:4621-4624)
            self.ctx.set_freeze_boundary(False)
        self.frame_count += 1
        if math.isfinite(self.E) and self.E < self.E_min:
            self.E_min = self.E
        if (not self.dynamics and self.convergence_threshold is None and not self.no_auto_dynamics
                and self.phase_steps >= 10000):
            self.dynamics = True
        if not self.dynamics and self.convergence_threshold is not None and self.phase_steps > 200:
            if self._prevE is not None and abs(self.E - self._prevE) < self.convergence_threshold and math.isfinite(self.E):
                self._conv_count += 1
                if self._conv_count >= 3:  # 3 consecutive frames within the threshold
                    self.phase = 1
                    self._conv_count = 0
                    self.converged_at = self.phase_steps
            else:
                self._conv_count = 0
            self._prevE = self.E
        if not self.dynamics and self.phase_steps >= self.total_steps:
            self.phase = 1
        return self.energies()

    def energies(self) -> Dict:
        return {k: getattr(self, k, None) for k in ("E", "E_T", "E_eK", "E_ee", "E_KK", "E_min", "phase_steps", "phase")}

    def _forces(self):
        """molecule.js:3205-3258: the GPU force per entry plus the softened repulsion of the unique
        nuclei (applied to every entry of a site); hinge atoms show no force."""
        F = self.ctx.forces(L.FORCE_GRADP)
        n, h = self.n, self.h
        self.nuc_force_elec = [[0.0] * 3 if (self.Z[a] == 0 and self.Z_nuc[a] == 0) else [float(v) for v in F[a]]
                               for a in range(n)]
        self.nuc_force_nuc = [[0.0, 0.0, 0.0] for _ in range(n)]
        if self.add_nuc_repulsion:
            for A in self.unique:
                ea = A["elec"][0]
                f = self._site_repulsion(A, ea)
                for e in A["elec"]:
                    self.nuc_force_nuc[e] = list(f)
        for a in range(n):
            if self.Z[a] == 0 and self.Z_nuc[a] == 0:
                continue
            self.nuc_force_total[a] = [self.nuc_force_elec[a][d] + self.nuc_force_nuc[a][d] for d in range(3)]
        for a in self.hinge_atoms:
            if a < n:
                self.nuc_force_total[a] = [0.0, 0.0, 0.0]

    def _site_repulsion(self, A, ea):
        fx = fy = fz = 0.0
        h = self.h
        for B in self.unique:
            if B is A:
                continue
            eb = B["elec"][0]
            dx = (self.pos[ea][0] - self.pos[eb][0]) * h
            dy = (self.pos[ea][1] - self.pos[eb][1]) * h
            dz = (self.pos[ea][2] - self.pos[eb][2]) * h
            r2 = dx * dx + dy * dy + dz * dz + h * h
            r = math.sqrt(r2)
            inv_r3 = 1.0 / (r * r2)
            q = A["Z_eff"] * B["Z_eff"]
            fx += q * dx * inv_r3
            fy += q * dy * inv_r3
            fz += q * dz * inv_r3
        return fx, fy, fz

    # ---- moveNuclei -------------------------------------------------------------------------------
    def move_nuclei(self):
        """moveNuclei (molecule.js:3742-4583) without the classical-MD backbone; then the warm K rebuild
        (the converged psi, labels and P are kept)."""
        n, h, NN = self.n, self.h, self.NN
        F = [[0.0] * 3 if self.Z[a] == 0 else list(self.nuc_force_elec[a]) for a in range(n)]
        if self.add_nuc_repulsion:
            for A in self.unique:
                f = self._site_repulsion(A, A["elec"][0])
                for e in A["elec"]:
                    F[e] = [F[e][0] + f[0], F[e][1] + f[1], F[e][2] + f[2]]
        if self.external_force:
            for a, f in enumerate(self.external_force[:n]):
                if f:
                    for d in range(3):
                        F[a][d] += f[d] or 0
                        self.nuc_force_total[a][d] += f[d] or 0
        for a in self.hinge_atoms:
            if a < n:
                F[a] = [0.0, 0.0, 0.0]
        if self.classical_md and self.classical_md.get("caIndices"):
            self.nuc_force = F
            self._classical_md(F)
            return
        pos = self.pos
        for i1, i2, r0, kb in self.bond_constraints:  # :4331-4346
            rx, ry, rz = ((pos[i1][d] - pos[i2][d]) * h for d in range(3))
            r = math.sqrt(rx * rx + ry * ry + rz * rz)
            if r < 1e-8:
                continue
            u = (rx / r, ry / r, rz / r)
            f = -kb * (r - r0)
            for d in range(3):
                F[i1][d] += f * u[d]
                F[i2][d] -= f * u[d]
        th0 = self.hoh_eq * math.pi / 180
        for o, h1, h2 in self.water_triplets:  # :4350-4385
            r1 = [(pos[h1][d] - pos[o][d]) * h for d in range(3)]
            r3 = [(pos[h2][d] - pos[o][d]) * h for d in range(3)]
            d1, d3 = math.sqrt(sum(x * x for x in r1)), math.sqrt(sum(x * x for x in r3))
            if d1 < 1e-6 or d3 < 1e-6:
                continue
            u1, u3 = [x / d1 for x in r1], [x / d3 for x in r3]
            cos = min(0.9999, max(-0.9999, u1[0] * u3[0] + u1[1] * u3[1] + u1[2] * u3[2]))
            th = math.acos(cos)
            s = math.sin(th)
            if s < 1e-6:
                continue
            c = self.bend_k * (th - th0) / s
            f1 = [c * (u3[d] - cos * u1[d]) / d1 for d in range(3)]
            f3 = [c * (u1[d] - cos * u3[d]) / d3 for d in range(3)]
            for d in range(3):
                F[h1][d] += f1[d]
                F[h2][d] += f3[d]
                F[o][d] -= f1[d] + f3[d]
        for grp in self.coincident_groups:  # :4390-4403
            g0 = grp[0]
            for gm in grp[1:]:
                for d in range(3):
                    F[g0][d] += F[gm][d]
                F[gm] = [0.0, 0.0, 0.0]
        self.nuc_force = F
        clamp = lambda x: max(5.0, min(NN - 5.0, x))
        for _ in range(self.substeps):
            if self.rigid_groups:
                for grp in self.rigid_groups:
                    g = [0.0, 0.0, 0.0]
                    M = 0.0
                    for a in grp:
                        if a >= n or self.Z[a] == 0:
                            continue
                        for d in range(3):
                            g[d] += F[a][d]
                        M += nuc_mass(self.Z[a])
                    if M == 0:
                        continue
                    v = self.nuc_vel[grp[0]]
                    for d in range(3):
                        v[d] += g[d] / M * self.dt_nuc * self.force_scale
                        if self.langevin_kT <= 0:
                            v[d] *= self.damping
                        v[d] = max(-self.max_vel, min(self.max_vel, v[d]))
                    for a in grp:
                        if a >= n or self.Z[a] == 0:
                            continue
                        for d in range(3):
                            pos[a][d] = clamp(pos[a][d] + v[d] * self.dt_nuc / h)
                continue
            movable = [a for a in range(n) if not (self.Z[a] == 0 and self.Z_nuc[a] == 0) and a not in self.frozen_atoms]
            yc = (sum(pos[a][1] for a in movable) / len(movable)) if (self.shear_rate and movable) else 0.0
            for a in movable:
                m = nuc_mass(self.Z_nuc[a] or self.Z[a])
                if self.shear_rate:
                    fs = m * self.shear_rate * (pos[a][1] - yc) * h
                    F[a][0] += fs
                    self.nuc_force_total[a][0] += fs
                if self.brownian:
                    drift = self.dt_nuc * self.force_scale / self.brownian_gamma
                    noise = math.sqrt(2 * max(self.langevin_kT, 0) * self.dt_nuc / self.brownian_gamma)
                    for d in range(3):
                        pos[a][d] = clamp(pos[a][d] + (F[a][d] * drift + noise * self.rng.standard_normal()) / h)
                else:
                    v = self.nuc_vel[a]
                    for d in range(3):
                        v[d] += F[a][d] / m * self.dt_nuc * self.force_scale
                        if self.langevin_kT <= 0:
                            v[d] *= self.damping
                        v[d] = max(-self.max_vel, min(self.max_vel, v[d]))
                        pos[a][d] = clamp(pos[a][d] + v[d] * self.dt_nuc / h)
            if self.langevin_kT > 0 and not self.brownian:  # Andersen collisions (:4495-4524)
                for a in movable:
                    if self.rng.random() < self.langevin_gamma:
                        m = nuc_mass(self.Z_nuc[a] or self.Z[a])
                        sv = math.sqrt(self.langevin_kT / m)
                        self.nuc_vel[a] = [sv * self.rng.standard_normal() for _ in range(3)]
                        sx = self.thermal_kick or (sv * self.dt_nuc / h)
                        for d in range(3):
                            pos[a][d] = clamp(pos[a][d] + sx * self.rng.standard_normal())
        for grp in self.coincident_groups:
            for gm in grp[1:]:
                pos[gm] = list(pos[grp[0]])
        self.nuc_steps += 1
        self._upload_atoms()

    def temperature(self) -> float:
        """The thermostat's kinetic temperature in K (molecule.js:4545-4556)."""
        ke, na = 0.0, 0
        for a in range(self.n):
            if (self.Z[a] == 0 and self.Z_nuc[a] == 0) or a in self.frozen_atoms:
                continue
            ke += 0.5 * nuc_mass(self.Z_nuc[a] or self.Z[a]) * sum(v * v for v in self.nuc_vel[a])
            na += 1
        return 2 * ke / (3 * na) * 315775 if na and ke > 0 else 0.0

    # ---- restarts ---------------------------------------------------------------------------------
    def restartWithPositions(self, new_positions):  # noqa: N802 -- molecule.js:2127-2149
        for e, p in enumerate(new_positions[:self.n]):
            self.pos[e] = [float(x) for x in p]
            self.mol_pos[e] = [float(x) for x in p]
        self._upload_atoms()
        self.initialize()

    def activateAtoms(self, count: int):  # noqa: N802 -- molecule.js:2151-2195
        count = max(1, min(int(count), self.n))
        self.Z = [self.Z_orig[e] if e < count else 0.0 for e in range(self.n)]
        self.nuc_vel = [[0.0, 0.0, 0.0] for _ in range(self.n)]
        self.nuc_force = [[0.0, 0.0, 0.0] for _ in range(self.n)]
        self.pos = [list(p) for p in self.mol_pos]
        self._upload_atoms()
        self.initialize()
        self.nuc_steps = 0
        self.active_count = count

    def extract(self, slice_k: Optional[int] = None) -> np.ndarray:
        """The page's slice buffer (extractWGSL, molecule.js:1108-1192)."""
        return self.ctx.extract(slice_k)

    def close(self):
        self.ctx.close()
