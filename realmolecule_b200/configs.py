"""Seeded synthetic workloads (the molecules and clusters the benchmarks run on).

Geometries are in bohr.  ``to_reference_atoms`` maps a geometry onto the reference's atom
list idiom (one entry per nucleus, domain charge Z = nuclear charge, all-electron, grid
units, cloud/solver.py:331-336); ``to_domain_atoms`` maps it onto the new flavour's idiom
(bare nuclei entries with Z = 0 and Z_nuc = charge, plus one unit-charge domain entry per
electron seed, molecule.js:12-17 / :50-67 style).

Workloads (name: what it is):
  h2o64      single H2O, 10 electrons, 64^3 at h = 0.25 bohr
  glycine128 glycine NH2-CH2-COOH, 10 atoms / 40 electrons, 128^3 at h = 0.2 bohr,
             seeded random rigid rotation
  clusters96 96 water clusters of 1-12 molecules, grids 48^3-128^3 at h = 0.25 bohr
  water100   100 waters (1000 electrons) at 1 g/cm^3, 192^3 at h = 0.2 bohr
  water1000  1000 waters (~10,000 electrons), 320^3 at h = 0.2 bohr
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Tuple

import numpy as np

ANG = 1.8897261246  # bohr per angstrom
Z_OF = {"H": 1, "C": 6, "N": 7, "O": 8}


@dataclass
class Geometry:
    name: str
    elements: List[str]
    xyz: np.ndarray                     # (n, 3) bohr, centred on the centroid
    NN: int
    h: float
    seeds: np.ndarray = field(default=None)  # (n_e, 3) bohr electron-domain seeds
    seed_owner: np.ndarray = field(default=None)

    @property
    def screen(self) -> float:
        return self.NN * self.h

    @property
    def charges(self) -> np.ndarray:
        return np.array([Z_OF[e] for e in self.elements], np.float64)


def _place(a, b, c, bond, angle_deg, dihedral_deg):
    """Natural-extension reference frame: position of d with |cd| = bond, angle bcd, dihedral abcd."""
    ang, dih = math.radians(angle_deg), math.radians(dihedral_deg)
    bc = c - b
    bc /= np.linalg.norm(bc)
    n = np.cross(b - a, bc)
    n /= np.linalg.norm(n)
    m = np.cross(n, bc)
    d2 = np.array([-bond * math.cos(ang), bond * math.sin(ang) * math.cos(dih), bond * math.sin(ang) * math.sin(dih)])
    return c + d2[0] * bc + d2[1] * m + d2[2] * n


def glycine_bohr() -> Tuple[List[str], np.ndarray]:
    """Glycine from standard internal coordinates (angstrom), trans backbone."""
    N = np.array([0.0, 0.0, 0.0])
    CA = np.array([1.47, 0.0, 0.0])
    tet = 109.47
    C = CA + 1.52 * np.array([-math.cos(math.radians(tet)), math.sin(math.radians(tet)), 0.0])
    O1 = _place(N, CA, C, 1.21, 120.0, 0.0)       # C=O
    O2 = _place(N, CA, C, 1.34, 120.0, 180.0)     # C-O(H), trans to N
    HO = _place(CA, C, O2, 0.97, tet, 180.0)
    HA1 = _place(C, N, CA, 1.09, tet, 120.0)
    HA2 = _place(C, N, CA, 1.09, tet, -120.0)
    HN1 = _place(C, CA, N, 1.01, tet, 60.0)
    HN2 = _place(C, CA, N, 1.01, tet, -60.0)
    el = ["N", "C", "C", "O", "O", "H", "H", "H", "H", "H"]
    xyz = np.stack([N, CA, C, O1, O2, HO, HA1, HA2, HN1, HN2]) * ANG
    return el, xyz


def random_rotation(rng) -> np.ndarray:
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q @ np.diag(np.sign(np.diag(r)))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def water_bohr(rot: np.ndarray) -> np.ndarray:
    """O, H, H of a rigid water (0.9572 A, 104.5 deg), rotated."""
    r, half = 0.9572 * ANG, math.radians(104.5) / 2
    local = np.array([[0, 0, 0], [r * math.sin(half), r * math.cos(half), 0], [-r * math.sin(half), r * math.cos(half), 0]])
    return local @ rot.T


def fibonacci_dirs(n: int) -> np.ndarray:
    k = np.arange(n) + 0.5
    phi = np.arccos(1 - 2 * k / n)
    th = math.pi * (1 + 5 ** 0.5) * k
    return np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], 1)


def electron_seeds(elements, xyz, rng, jitter=0.05):
    """Per atom: H -> 1 seed at the nucleus; heavy atom with Z electrons -> 2 core seeds at the
    nucleus and Z-2 valence seeds on an r = 1.2 bohr sphere (Fibonacci directions); every seed
    jittered by N(0, jitter) bohr.  Returns (seeds, owner atom index)."""
    seeds, owner = [], []
    for a, (e, p) in enumerate(zip(elements, xyz)):
        z = Z_OF[e]
        if z == 1:
            pts = [p]
        else:
            pts = [p, p] + [p + 1.2 * d for d in fibonacci_dirs(z - 2)]
        for q in pts:
            seeds.append(q + rng.normal(0, jitter, 3))
            owner.append(a)
    return np.array(seeds), np.array(owner)


def h2o64(seed: int = 0) -> Geometry:
    xyz = np.array([[0.0, 0.0, 0.0], [1.4305, 1.1078, 0.0], [-1.4305, 1.1078, 0.0]])
    xyz -= xyz.mean(0)
    g = Geometry("h2o64", ["O", "H", "H"], xyz, 64, 0.25)
    g.seeds, g.seed_owner = electron_seeds(g.elements, g.xyz, np.random.default_rng(seed))
    return g


def glycine128(seed: int = 0) -> Geometry:
    rng = np.random.default_rng(seed)
    el, xyz = glycine_bohr()
    xyz = (xyz - xyz.mean(0)) @ random_rotation(rng).T
    g = Geometry("glycine128", el, xyz, 128, 0.2)
    g.seeds, g.seed_owner = electron_seeds(el, xyz, rng)
    return g


def water_box(n_mol: int, edge: float, min_oo_ang: float, rng, sphere=False, max_tries=200000):
    """Rejection-sample n_mol rigid waters with random orientation; O-O >= min_oo."""
    O = []
    mols = []
    tries = 0
    while len(mols) < n_mol:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place waters")
        if sphere:
            p = rng.uniform(-edge, edge, 3)
            if np.linalg.norm(p) > edge:
                continue
        else:
            p = rng.uniform(-edge / 2, edge / 2, 3)
        if O and np.min(np.linalg.norm(np.array(O) - p, axis=1)) < min_oo_ang * ANG:
            continue
        O.append(p)
        mols.append(water_bohr(random_rotation(rng)) + p)
    xyz = np.concatenate(mols)
    return ["O", "H", "H"] * n_mol, xyz - xyz.mean(0)


def water_cluster_grid(xyz, h, margin=6.0, multiple=16, lo=48, hi=128):
    ext = float(np.max(np.abs(xyz))) * 2 + 2 * margin
    NN = int(math.ceil(ext / h / multiple) * multiple)
    return max(lo, min(hi, NN))


def clusters96(seed: int = 0, n_inst: int = 96) -> List[Geometry]:
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n_inst):
        n = int(rng.integers(1, 13))
        radius = 2.0 * ANG * (n ** (1 / 3)) + 1.0
        el, xyz = water_box(n, radius, 2.7, rng, sphere=True)
        NN = water_cluster_grid(xyz, 0.25)
        g = Geometry(f"cluster{q}", el, xyz, NN, 0.25)
        g.seeds, g.seed_owner = electron_seeds(el, xyz, rng)
        out.append(g)
    return out


def water100(seed: int = 0) -> Geometry:
    rng = np.random.default_rng(seed)
    el, xyz = water_box(100, 27.2, 2.5, rng)
    g = Geometry("water100", el, xyz, 192, 0.2)
    g.seeds, g.seed_owner = electron_seeds(el, xyz, rng)
    return g


def water1000(seed: int = 0) -> Geometry:
    rng = np.random.default_rng(seed)
    el, xyz = water_box(1000, 58.6, 2.5, rng)
    g = Geometry("water1000", el, xyz, 320, 0.2)
    g.seeds, g.seed_owner = electron_seeds(el, xyz, rng)
    return g


def to_reference_atoms(g: Geometry, rc: dict | None = None) -> List[dict]:
    """Reference idiom: one entry per nucleus at grid position x/h + NN/2, Z = nuclear charge."""
    N2 = g.NN // 2
    rows = []
    for e, p in zip(g.elements, g.xyz):
        z = float(Z_OF[e])
        rows.append({"i": float(p[0] / g.h + N2), "j": float(p[1] / g.h + N2), "k": float(p[2] / g.h + N2),
                     "Z": z, "Z_nuc": z, "rc": float((rc or {}).get(e, 0.0)), "el": e})
    return rows


def to_domain_atoms(g: Geometry) -> List[dict]:
    """New-flavour idiom: nuclei as bare entries (Z = 0, Z_nuc = charge), then one unit domain
    per electron seed (Z = 1, Z_nuc = 0)."""
    N2 = g.NN // 2
    rows = [{"i": float(p[0] / g.h + N2), "j": float(p[1] / g.h + N2), "k": float(p[2] / g.h + N2), "Z": 0.0,
             "Z_nuc": float(Z_OF[e]), "el": e} for e, p in zip(g.elements, g.xyz)]
    for s in g.seeds:
        rows.append({"i": float(s[0] / g.h + N2), "j": float(s[1] / g.h + N2), "k": float(s[2] / g.h + N2),
                     "Z": 1.0, "Z_nuc": 0.0, "el": ""})
    return rows


def reference_config(g: Geometry, **extra) -> dict:
    """cloud/solver.py config dict for a geometry (valence-free, all-electron idiom)."""
    cfg = {"gridN": g.NN, "screen": g.screen, "atoms": to_reference_atoms(g)}
    cfg.update(extra)
    return cfg


def _js_round(x: float) -> int:
    """JavaScript's Math.round (halves round up)."""
    return math.floor(x + 0.5)


def mol_fast_h2_page(sep: float = 1.4) -> dict:
    """The H2 page of mol_fast.js (mol_fast_h2.html:16-33): NN = 200, 10 bohr box, the two nuclei
    sep apart on the i axis, dynamics on.  Keyword arguments of ``MolFast``."""
    N, scr = 200, 10.0
    h, N2 = scr / N, _js_round(N / 2)
    di = _js_round(sep / h / 2)
    return {"nuclei": [{"i": N2 - di, "j": N2, "k": N2, "Z": 1, "rc": 0.0, "z_init": 1.0},
                       {"i": N2 + di, "j": N2, "k": N2, "Z": 1, "rc": 0.0, "z_init": 1.0}],
            "NN": N, "screen": scr, "norm_targets": [1, 1], "max_steps": 50000, "dynamics": True}


def mol_fast_ch4_page(bond: float = 2.054, scr: float = 12.0) -> dict:
    """The CH4 page of mol_fast.js (mol_fast_ch4.html:18-54): NN = 200, a Z = 4 carbon pseudo-atom
    (rc 0.5, one 4-electron orbital) at the centre and four tetrahedral H at `bond` bohr, grid-rounded;
    dynamics on.  Keyword arguments of ``MolFast``."""
    N = 200
    h, N2 = scr / N, _js_round(N / 2)

    def shift(dx, dy, dz):
        return {"i": _js_round(N2 + dx * bond / h), "j": _js_round(N2 + dy * bond / h),
                "k": _js_round(N2 + dz * bond / h)}

    s2, s6 = math.sqrt(2), math.sqrt(6)
    hs = [shift(1, 0, 0), shift(-1 / 3, 2 * s2 / 3, 0), shift(-1 / 3, -s2 / 3, s6 / 3), shift(-1 / 3, -s2 / 3, -s6 / 3)]
    nuc = [{"i": N2, "j": N2, "k": N2, "Z": 4, "rc": 0.5}] + [dict(x, Z=1, rc=0.0) for x in hs]
    return {"nuclei": nuc, "NN": N, "screen": scr, "norm_targets": [4, 1, 1, 1, 1], "max_steps": 100000,
            "alpha_tf": 0.0, "dynamics": True}


def realqm_rb_h2_page(sep: float = 1.4) -> dict:
    """The direct H2 page of realqm_rb.js (h2_rb_direct.html:12-31): NN = 100, 8 bohr box, the
    nuclei sep apart on the i axis, one electron each.  Keyword arguments of ``RealqmRb``."""
    N, scr = 100, 8.0
    h, N2 = scr / N, _js_round(N / 2)
    dI = _js_round(sep / h / 2)
    return {"nuclei": [{"i": N2 - dI, "j": N2, "k": N2, "Z": 1, "rc": 0, "ne": 1},
                       {"i": N2 + dI, "j": N2, "k": N2, "Z": 1, "rc": 0, "ne": 1}],
            "NN": N, "screen": scr, "nelec": 2, "norm_targets": [1, 1], "max_steps": 30000}


WORKLOADS = {"h2o64": h2o64, "glycine128": glycine128, "water100": water100, "water1000": water1000}
