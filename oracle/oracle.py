"""Python face of the oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
may import this module.  It provides

* ``build()``            -- compile oracle/rq_oracle.c (and, when the reference tree is
                            present, the reference kernels via oracle/ref_build.py);
* ``O``                  -- numpy wrappers over the C restatement (oracle/rq_oracle.c);
* ``RefKernels``         -- numpy wrappers over the reference's own cloud/solver.py
                            kernels compiled for the host (oracle/_ref/libsolverpy_ref.so);
* ``SolverPyDriver``     -- the schedule of ``RealQMSolver.run`` (cloud/solver.py:402-634)
                            restated over either kernel set, used as the CPU baseline and
                            as the multi-step oracle of the solver.py flavour.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SRC = os.path.join(HERE, "rq_oracle.c")
ORACLE_LIB = os.path.join(HERE, "librq_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libsolverpy_ref.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i, _i64, _f, _d = C.c_int, C.c_int64, C.c_float, C.c_double


def build(force: bool = False, with_reference: bool = True) -> None:
    """Compile the C oracle (and the reference kernels when the reference tree exists)."""
    if force or not os.path.exists(ORACLE_LIB) or os.path.getmtime(ORACLE_LIB) < os.path.getmtime(ORACLE_SRC):
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
                               "-fno-fast-math", ORACLE_SRC, "-o", ORACLE_LIB, "-lm"])
    if with_reference:
        import importlib.util
        spec = importlib.util.spec_from_file_location("rq_ref_build", os.path.join(HERE, "ref_build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        try:
            mod.build(quiet=True)
        except FileNotFoundError:
            pass  # no reference tree and no prebuilt library: reference-pinned tests skip


class MjAtom(C.Structure):
    """molecule.js atom record (molecule.js:183-191) as the oracle takes it."""
    _fields_ = [("posI", C.c_uint32), ("posJ", C.c_uint32), ("posK", C.c_uint32), ("Z", C.c_float),
                ("rc", C.c_float), ("Z_nuc", C.c_float), ("initZeff", C.c_float), ("initRcut", C.c_float)]


class MjSplit(C.Structure):
    """Shell split of one entry (molecule.js:183-191 split fields) as the oracle takes it."""
    _fields_ = [("type", C.c_uint32), ("idx", C.c_uint32), ("ax", C.c_float), ("ay", C.c_float), ("az", C.c_float),
                ("rot", C.c_float)]


SPLIT_CODES = {"sphere": 0, "hemi": 2, "third": 3, "tetra": 4}  # fillAtomBuf's stCode (molecule.js:1894)


def mj_atoms(rows):
    """rows: iterable of dicts with i,j,k,Z[,rc,Z_nuc,initZeff,initRcut] -> ctypes array.

    Positions are truncated to unsigned integers like molecule.js:1882-1884."""
    rows = list(rows)
    arr = (MjAtom * len(rows))()
    for n, a in enumerate(rows):
        arr[n].posI, arr[n].posJ, arr[n].posK = int(a["i"]), int(a["j"]), int(a["k"])
        arr[n].Z = a["Z"]
        arr[n].rc = a.get("rc", 0.0)
        arr[n].Z_nuc = a.get("Z_nuc", a["Z"])
        arr[n].initZeff = a.get("initZeff", a["Z"]) or a["Z"]
        arr[n].initRcut = a.get("initRcut", 1e6)
    return arr


class _Oracle:
    def __init__(self):
        build(with_reference=False)
        L = C.CDLL(ORACLE_LIB)
        sig = {
            "orc_sp_init_trial": [_f32p, _i32p, _f32p, _f32p, _f32p, _i, _i, _f, _f],
            "orc_sp_recompute_K": [_f32p, _f32p, _i, _i, _f, _f],
            "orc_sp_update": [_f32p, _f32p, _f32p, _f32p, _i32p, _i, _f, _f],
            "orc_sp_boundary_snapshot": [_i32p, _i32p, _f32p, _i, _i, _f, _f],
            "orc_sp_boundary_inplace_lex": [_i32p, _f32p, _i, _i, _f, _f],
            "orc_sp_jacobi": [_f32p, _f32p, _f32p, _i, _f, _f],
            "orc_sp_norms_f32_seq": [_f32p, _i32p, _i64, _i, _f, _f32p],
            "orc_sp_norms_f64": [_f32p, _i32p, _i, _i, _d, _f64p],
            "orc_sp_normalize": [_f32p, _i32p, _f32p, _f32p, _i64, _i],
            "orc_sp_energy_blocktree": [_f32p, _f32p, _f32p, _i32p, _f32p, _i, _f, _f, _i],
            "orc_sp_energy_f64": [_f32p, _f32p, _f32p, _i32p, _i, _d, _d, _f64p, _i, C.c_void_p],
            "orc_sp_forces": [_f32p, _f32p, _i, _i, _f, _f, _f, _f64p],
            "orc_mj_update": [_f32p, _f32p, _f32p, _u32p, _f32p, C.c_void_p, _i, _i, _i, _f, _f, _f],
            "orc_mj_evolve_boundary": [_u32p, _u32p, _f32p, _f32p, _i, _f, _f, C.c_void_p, C.c_void_p, C.c_void_p,
                                       _f],
            "orc_mj_jacobi": [_f32p, _f32p, _f32p, _i, _f, _f],
            "orc_mj_rho": [_f32p, _f32p, _i],
            "orc_mj_rho_self": [_f32p, _u32p, C.c_uint32, _f32p, _i],
            "orc_mj_rho_other": [_f32p, _u32p, C.c_uint32, _f32p, _i],
            "orc_mj_copy_for_label": [_f32p, _f32p, _u32p, C.c_uint32, _i],
            "orc_mj_init_pdirect": [C.c_void_p, _i, C.c_uint32, _f32p, _f32p, _i, _f, _f],
            "orc_mj_sub_self": [_f32p, _f32p, _u32p, C.c_uint32, _f, _i],
            "orc_mj_update_cheb": [_f32p, _f32p, _f32p, _u32p, _f32p, C.c_void_p, _i, _i, _f, _f, _f, _f],
            "orc_mj_residual": [_f32p, _f32p, _f32p, _i, _f, _f],
            "orc_mj_restrict": [_f32p, _f32p, _i, _i],
            "orc_mj_coarse_smooth": [_f32p, _f32p, _f32p, _i, _f],
            "orc_mj_prolong": [_f32p, _f32p, _i, _i],
            "orc_mj_norms_fixed": [_f32p, _u32p, _i, _f, _i, _u32p, _f32p],
            "orc_mj_normalize": [_f32p, _f32p, _u32p, C.c_void_p, _i],
            "orc_mj_energy": [_f32p, _f32p, _f32p, _u32p, C.c_void_p, _i, _f, _f, _f, _f64p],
            "orc_mj_force_gradP": [_f32p, C.c_void_p, _i, _i, _f, _i, _f64p],
            "orc_mj_force_hf": [_f32p, C.c_void_p, _i, _i, _f, _f, _f64p],
            "orc_mj_init": [_f32p, _f32p, _u32p, C.c_void_p, _i, _i, _f, _f, _f, C.c_void_p],
            "orc_mj_init_persist": [_f32p, _f32p, _u32p, C.c_void_p, _i, _i, _f, _f, _f, C.c_void_p],
            "orc_mj_recompute_k": [_f32p, C.c_void_p, _i, _i, _f, _f],
            "orc_nm_potential": [_f64p, _f64p, _f64p, _i, _i, _d, _d],
            "orc_nm_update": [_f64p, _f64p, _f64p, _f64p, _i32p, _i, _d, _d],
            "orc_nm_vcycle": [_f64p, _f64p, _i, _d, _i, _i, _i, _i],
            "orc_nm_energy": [_f64p, _f64p, _f64p, _i32p, _i, _d, _f64p, _i, _f64p],
            "orc_nm_normalize": [_f64p, _i32p, _i64, _i, _f64p, _f64p],
            "orc_nm_force": [_f64p, _f64p, _f64p, _i, _i, _d, _d, _f64p],
            "orc_nm_init": [_f64p, _i32p, _f32p, _i32p, _i, _i, _f],
            "orc_nm_evolve": [_i32p, _i32p, _f64p, _f32p, _i, _d, _d],
            "orc_nm_evolve_f32": [_i32p, _i32p, _f32p, _f32p, _i, _f, _f],
            "orc_at_init": [_f32p, _f32p, _f32p, _f32p, C.c_void_p, _i, _i, _d, _d],
            "orc_at_step": [_f32p, _f32p, _f32p, _f32p, C.c_void_p, _i, _i, _d, _d, _i, _f64p, _f64p],
            "orc_mf_update": [C.c_void_p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p],
            "orc_mf_reduce": [C.c_void_p, _f32p, _f32p, _f32p, _f32p, _f32p],
            "orc_mf_normalize": [C.c_void_p, _f32p, _f32p],
            "orc_mf_vcycle": [C.c_void_p, _f32p, _f32p, _i, _i],
            "orc_mf_force": [C.c_void_p, _f32p, _f32p],
            "orc_mf_recompute_k": [C.c_void_p, _f32p],
            "orc_mf_extract": [C.c_void_p, _f32p, _f32p, _f32p, _f32p],
            "orc_mf_init": [_i, _d, _i, _f64p, _f32p, _f32p, _f32p, _f32p],
            "orc_rb_rho_nearest": [C.c_void_p, _f32p, _f32p, _f32p],
            "orc_rb_wu": [C.c_void_p, _i, _i, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p],
            "orc_rb_p": [C.c_void_p, _i, _i, _f32p, _f32p, _f32p],
            "orc_rb_normalize": [C.c_void_p, _i, _f32p],
            "orc_rb_energy": [C.c_void_p, _f32p, _f32p, _f32p, _f32p, _d, _d, _f64p],
            "orc_rb_init": [C.c_void_p, _i, _f32p, _i32p, _f32p, _f32p, _f32p, _f32p],
            "orc_rb_slice": [C.c_void_p, _f32p, _f32p, _f32p, _f32p, _f32p],
            "orc_lob_apply_h": [_f32p, _f32p, _f32p, _u32p, _f32p, C.c_void_p, _i, _f, _f],
            "orc_lob_inner": [_f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _u32p, C.c_uint32, _i, _f, _f32p],
            "orc_lob_residual": [_f32p, _f32p, _f32p, _u32p, _f32p, _f32p, _f, C.c_uint32, _i, _f],
            "orc_lob_update": [_f32p, _f32p, _f32p, _u32p, _f, _f, _f, C.c_uint32, _i],
            "orc_lob_ritz2": [_f64p, _f64p],
            "orc_lob_ritz3": [_f64p, _f64p],
        }
        for name, argt in sig.items():
            fn = getattr(L, name)
            fn.argtypes = argt
            fn.restype = None
            setattr(self, name[4:], fn)
        L.orc_rb_normalize.restype = C.c_float
        self.lib = L


_O = None


def O() -> _Oracle:
    """The loaded C oracle (compiled on first use)."""
    global _O
    if _O is None:
        _O = _Oracle()
    return _O


class RefKernels:
    """The reference's own cloud/solver.py kernels compiled for the host (oracle/_ref)."""

    SIGS = {
        "initTrial": ["p", "p", "p", "p", "p", "i", "i", "f", "f"],
        "updateU": ["p", "p", "p", "p", "p", "i", "f", "f"],
        "boundaryEvolve": ["p", "p", "p", "i", "i", "f", "f", "f", "f"],
        "recomputeK": ["p", "p", "i", "i", "f", "f"],
        "computeRho": ["p", "p", "i"],
        "jacobiStep": ["p", "p", "p", "i", "f", "f"],
        "normalizeU": ["p", "p", "p", "p", "i", "i", "f"],
        "computeForceAll": ["p", "p", "p", "i", "i", "f", "f", "f"],
    }

    def __init__(self, path: str = REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        tmap = {"p": C.c_void_p, "i": C.c_int, "f": C.c_float}
        for name, s in self.SIGS.items():
            for pre in ("rqref_launch_", "rqref_launch_serial_"):
                fn = getattr(self.lib, pre + name)
                fn.argtypes = [C.c_int, C.c_int] + [tmap[c] for c in s]
                fn.restype = None

    def launch(self, name, grid, block, args, serial=False):
        conv = []
        for a in args:
            if isinstance(a, np.ndarray):
                assert a.flags.c_contiguous
                conv.append(a.ctypes.data)
            elif isinstance(a, (np.floating, float)):
                conv.append(float(a))
            else:
                conv.append(int(a))
        fn = getattr(self.lib, ("rqref_launch_serial_" if serial else "rqref_launch_") + name)
        fn(int(grid), int(block), *conv)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def solverpy_dv(n_elec: int) -> float:
    """Time-step table of cloud/solver.py:342-351."""
    if n_elec > 500:
        return 0.005
    if n_elec > 200:
        return 0.01
    if n_elec > 100:
        return 0.02
    if n_elec > 30:
        return 0.03
    return 0.12


class SolverPyDriver:
    """Restatement of the RealQMSolver state and schedule (cloud/solver.py:321-634).

    ``kernels="reference"`` runs the reference's own kernels (oracle/_ref) with
    numpy norms exactly as the reference host code computes them (f32 np.add.at);
    ``kernels="oracle"`` runs the C restatement with FP64 per-domain norms, which is
    the arithmetic the CUDA product uses.  Dynamics are not restated here.
    """

    def __init__(self, config: dict, kernels: str = "oracle", label_mode: str = "snapshot"):
        self.label_mode = label_mode
        self.NN = int(config["gridN"])
        self.S = self.NN + 1
        self.S3 = self.S ** 3
        self.h = config["screen"] / self.NN
        self.h2 = self.h * self.h
        self.h3 = self.h ** 3
        N2 = self.NN // 2
        atoms = config["atoms"]
        self.nAtoms = len(atoms)
        self.Z_eff = np.array([a["Z"] for a in atoms], dtype=np.float32)
        self.atom_pos = np.array([[a["i"], a["j"], a.get("k", N2)] for a in atoms], dtype=np.float32)
        self.atom_rc = np.array([a.get("rc", 0) for a in atoms], dtype=np.float32)
        self.nElec = int((self.Z_eff > 0).sum())
        self.dv = float(config.get("dv", solverpy_dv(self.nElec)))
        self.half_dv = 0.5 * self.dv
        self.dtv = self.dv * self.h2
        self.U = np.zeros(self.S3, np.float32)
        self.U2 = np.zeros(self.S3, np.float32)
        self.K = np.zeros(self.S3, np.float32)
        self.P = np.zeros(self.S3, np.float32)
        self.P2 = np.zeros(self.S3, np.float32)
        self.rho = np.zeros(self.S3, np.float32)
        self.label = np.zeros(self.S3, np.int32)
        self.label2 = np.zeros(self.S3, np.int32)
        self.bestU = np.zeros(self.S3, np.float32)
        self.atoms5 = np.zeros((self.nAtoms, 5), np.float32)
        for n, a in enumerate(atoms):
            self.atoms5[n] = [a["i"], a["j"], a.get("k", N2), a["Z"], a.get("rc", 0)]
        self.atoms5 = np.ascontiguousarray(self.atoms5.reshape(-1))
        self.kernels = kernels
        self.block = 256
        self.grid = (self.S3 + self.block - 1) // self.block
        self.R = RefKernels() if kernels == "reference" else None
        self.E = self.E_T = self.E_eK = self.E_ee = self.E_KK = 0.0
        self.steps_done = 0

    # -- kernels ---------------------------------------------------------
    def initialize(self, bootstrap: int = 100):
        if self.R:
            self.R.launch("initTrial", self.grid, self.block,
                          (self.U, self.label, self.K, self.bestU, self.atoms5, self.nAtoms, self.S,
                           np.float32(self.h), np.float32(self.h2)))
        else:
            O().sp_init_trial(self.U, self.label, self.K, self.bestU, self.atoms5, self.nAtoms, self.S,
                              self.h, self.h2)
        self.normalize()
        for _ in range(bootstrap):
            self.poisson_step()

    def normalize(self):
        if self.R:
            norms = np.zeros(self.nAtoms, np.float32)
            O().sp_norms_f32_seq(self.U, self.label, self.S3, self.nAtoms, np.float32(self.h3), norms)
        else:
            n64 = np.zeros(self.nAtoms, np.float64)
            O().sp_norms_f64(self.U, self.label, self.S, self.nAtoms, self.h3, n64)
            norms = n64.astype(np.float32)
        if self.R:
            self.R.launch("normalizeU", self.grid, self.block,
                          (self.U, self.label, norms, self.Z_eff, self.S3, self.nAtoms, np.float32(self.h3)))
        else:
            O().sp_normalize(self.U, self.label, norms, self.Z_eff, self.S3, self.nAtoms)

    def poisson_step(self):
        coeff = np.float32(2.0 * np.pi)
        if self.R:
            self.R.launch("computeRho", self.grid, self.block, (self.rho, self.U, self.S3))
            for _ in range(2):
                self.R.launch("jacobiStep", self.grid, self.block,
                              (self.P, self.P2, self.rho, self.S, np.float32(self.h2), coeff))
                self.P, self.P2 = self.P2, self.P
        else:
            for _ in range(2):
                O().sp_jacobi(self.P, self.P2, self.U, self.S, self.h2, coeff)
                self.P, self.P2 = self.P2, self.P

    def update(self):
        if self.R:
            self.R.launch("updateU", self.grid, self.block,
                          (self.U, self.U2, self.K, self.P, self.label, self.S, np.float32(self.half_dv),
                           np.float32(self.dtv)))
        else:
            O().sp_update(self.U, self.U2, self.K, self.P, self.label, self.S, self.half_dv, self.dtv)
        self.U, self.U2 = self.U2, self.U

    def boundary(self):
        # snapshot semantics by default (the reference writes in place, which races on a
        # GPU); "inplace_lex" reproduces the reference kernel run serially in index order
        if self.label_mode == "inplace_lex":
            O().sp_boundary_inplace_lex(self.label, self.atoms5, self.nAtoms, self.S, self.h, self.h2)
            return
        O().sp_boundary_snapshot(self.label, self.label2, self.atoms5, self.nAtoms, self.S, self.h, self.h2)
        self.label, self.label2 = self.label2, self.label

    def step(self, step: int, norm_interval=20, poisson_interval=2):
        if step % poisson_interval == 0:
            self.poisson_step()
        self.update()
        if step % norm_interval == 0:
            self.normalize()
        if step % (norm_interval * 5) == 0:
            self.boundary()

    def run(self, total_steps: int, norm_interval=20, poisson_interval=2):
        """Continue the schedule for total_steps (the step counter persists across calls)."""
        for _ in range(total_steps):
            self.steps_done += 1
            self.step(self.steps_done, norm_interval, poisson_interval)

    def energy(self):
        out = np.zeros(3, np.float64)
        O().sp_energy_f64(self.U, self.K, self.P, self.label, self.S, self.h, self.h3, out, 0, None)
        self.E_T, self.E_eK, self.E_ee = map(float, out)
        self.E_KK = e_kk_solverpy(self.atom_pos, self.Z_eff, self.h)
        self.E = self.E_T + self.E_eK + self.E_ee + self.E_KK
        return self.E


def e_kk_solverpy(atom_pos, Z_eff, h) -> float:
    """cloud/solver.py:462-474: sum Za Zb / sqrt(d^2 + h^2) over active pairs (FP64)."""
    e = 0.0
    n = len(Z_eff)
    for a in range(n):
        if Z_eff[a] <= 0:
            continue
        for b in range(a + 1, n):
            if Z_eff[b] <= 0:
                continue
            d = (np.asarray(atom_pos[a], np.float64) - np.asarray(atom_pos[b], np.float64)) * h
            e += float(Z_eff[a]) * float(Z_eff[b]) / math.sqrt(float(d @ d) + h * h)
    return e


class MoleculeJsDriver:
    """Restatement of molecule.js's doSteps schedule (molecule.js:2822-3104) over the C oracle,
    total-Poisson path without SIC (the reference's choice for NELEC > 30), W_CUTOFF = 0, no
    locked groups or shell splits.  One ``step()`` is one iteration of doSteps' s-loop; every
    ``steps_per_frame`` steps the frame tail runs (Pother <- P, then the level-set passes).

    Parameters are the f32 values of the uniform buffer (molecule.js:1829-1836): h, h2 = f32(h*h
    in double), h3, 1/h^2, dt = f32(dv*h^2), half_d = f32(dv/2).
    """

    def __init__(self, NN, screen, atoms, dv=None, steps_per_frame=None, norm_interval=20, vcycle_interval=50,
                 jacobi_per_step=2, boundary_speed=0.5, curv_reg=0.15, sic=False, chebyshev=False, lobpcg=False,
                 locked_groups=None, splits=None):
        self.NN = NN
        self.S = NN + 1
        self.S3 = self.S ** 3
        h = screen / NN
        self.hd = h
        self.h = np.float32(h)
        self.h2 = np.float32(h * h)
        self.h3 = np.float32(h * h * h)
        self.inv_h2 = np.float32(1.0 / (h * h))
        self.Rsing = np.float32(2 * h)
        self.rows = [dict(a) for a in atoms]
        for r in self.rows:
            r.setdefault("Z_nuc", r["Z"])
        self.atoms = mj_atoms(self.rows)
        self.nA = len(self.rows)
        nelec = sum(1 for a in self.rows if a["Z"] > 0 or a.get("Z_nuc", 0) > 0)
        self.nelec = nelec
        self.n_electrons = sum(a["Z"] for a in self.rows)
        self.has_bare = any(a["Z"] == 0 and a.get("Z_nuc", 0) > 0 for a in self.rows)
        self.dv = dv if dv else (0.01 if nelec > 500 else 0.03 if nelec > 100 else 0.12)
        self.dt = np.float32(self.dv * h * h)
        self.half_d = np.float32(0.5 * self.dv)
        self.spf = steps_per_frame or (50 if nelec <= 30 else 5 if nelec <= 100 else 2)
        self.norm_interval, self.vcycle_interval, self.jps = norm_interval, vcycle_interval, jacobi_per_step
        self.dt_w, self.curv = np.float32(boundary_speed), np.float32(curv_reg)
        S3 = self.S3
        self.K = np.zeros(S3, np.float32)
        self.U = np.zeros(S3, np.float32)
        self.Unext = np.zeros(S3, np.float32)
        self.label = np.zeros(S3, np.uint32)
        self.label2 = np.zeros(S3, np.uint32)
        self.bestU = np.zeros(S3, np.float32)
        self.P = np.zeros(S3, np.float32)
        self.P2 = np.zeros(S3, np.float32)
        self.Pother = np.zeros(S3, np.float32)
        self.W = np.ones(S3, np.float32)
        self.rho = np.zeros(S3, np.float32)
        self.steps_done = 0
        self.frame = 0  # molecule.js frameCount
        self.chebyshev = bool(chebyshev)
        self.cheb_state, self.cheb_E = 1.0, 0.0  # chebOmega (:1762) and the page's E (:1767)
        # USER_LOCKED_GROUPS (molecule.js:490-503) as the bit set of each label's groups
        self.lock = np.zeros(self.nA, np.uint64)
        for g, members in enumerate(locked_groups or []):
            for mbr in members:
                self.lock[int(mbr)] |= np.uint64(1) << np.uint64(g)
        # shell splits per entry (USER_SPLIT_*, molecule.js:27-32): dicts of type, idx, axis, rot
        self.set_splits(splits)
        # useLOBPCG (molecule.js:1751): one step() is one doLOBPCGStep frame
        self.lobpcg = bool(lobpcg)
        self.sic = bool(sic)
        self.freeze = False  # window.FREEZE_BOUNDARY (molecule.js:3095, :3643)
        if self.lobpcg:
            self.HX, self.LW, self.HW, self.LP, self.HP = (np.zeros(S3, np.float32) for _ in range(5))
        # SIC_INTERVAL (molecule.js:112); 0 = off
        nel = nelec or 3
        # sic=True takes the reference's own Pother path: the direct per-electron Poisson for
        # NELEC <= 5 (USE_DIRECT_POTHER, molecule.js:111), else the SIC every SIC_INTERVAL frames
        self.direct = bool(sic) and nel <= 5
        self.sic_interval = (1 if nel <= 15 else 5 if nel <= 30 else 0) if sic and not self.direct else 0
        self.Pdirect = {}
        SC = NN // 2 + 1
        self.SC = SC

    def initialize(self, init_pos=None):
        """uploadInitialData (molecule.js:1905-2101).  init_pos: window.USER_INIT_POS, per entry an
        (i, j) or None -- the trial psi and labels are built with those entries moved there (k kept,
        :1909-1921), then K is rebuilt from 0 by recomputeK at the true positions (:1959-1981)."""
        moved = self.atoms
        if init_pos:
            rows = [dict(r) for r in self.rows]
            for n, p in enumerate(init_pos):
                if p is not None and n < len(rows):
                    rows[n]["i"], rows[n]["j"] = p[0], p[1]
            moved = mj_atoms(rows)
        O().mj_init(self.K, self.U, self.label, C.addressof(moved), self.nA, self.S, self.h, self.h2, self.Rsing,
                    self._splits_ptr())
        if init_pos:
            O().mj_recompute_k(self.K, C.addressof(self.atoms), self.nA, self.S, self.h, self.Rsing)
        self.bestU[:] = self.U
        self.Unext[:] = self.U
        self.label2[:] = self.label
        if self.direct and self.n_electrons > 1:  # molecule.js:2678-2693
            self.Pother[:] = 0
            for m, r in enumerate(self.rows):
                if np.float32(r["Z"]) == 0:
                    continue
                self.Pdirect[m] = np.zeros(self.S3, np.float32)
                O().mj_init_pdirect(C.addressof(self.atoms), self.nA, m, self.Pdirect[m], self.Pother, self.S, self.h,
                                    self.h2)

    def restart(self):
        """The classical-MD backbone's full restart (molecule.js:4236-4286): K, labels and the trial
        psi from scratch at the current positions, P cleared, W and Pother kept."""
        O().mj_init(self.K, self.U, self.label, C.addressof(self.atoms), self.nA, self.S, self.h, self.h2, self.Rsing,
                    self._splits_ptr())
        self.bestU[:] = self.U
        self.Unext[:] = self.U
        self.P[:] = 0
        self.P2[:] = 0

    def set_splits(self, splits):
        self.splits = None
        if splits:
            self.splits = (MjSplit * self.nA)()
            for n, sp in enumerate(splits):
                if not sp:
                    continue
                t = sp.get("type", 0)  # fillAtomBuf: a name through stCode, else the number (:1894-1896)
                self.splits[n].type = SPLIT_CODES.get(t, 0) if isinstance(t, str) else int(t or 0)
                self.splits[n].idx = int(sp.get("idx", 0))
                ax = sp.get("axis") or (0.0, 0.0, 1.0)
                self.splits[n].ax, self.splits[n].ay, self.splits[n].az = (float(v) for v in ax)
                self.splits[n].rot = float(sp.get("rot", 0.0))

    def _splits_ptr(self):
        return C.addressof(self.splits) if self.splits is not None else None

    def set_positions(self, rows):
        self.rows = [dict(a) for a in rows]
        for r in self.rows:
            r.setdefault("Z_nuc", r["Z"])
        self.atoms = mj_atoms(self.rows)
        O().mj_init_persist(self.K, self.bestU, self.label, C.addressof(self.atoms), self.nA, self.S, self.h, self.h2,
                            self.Rsing, self._splits_ptr())  # labelBuf only; label2Buf keeps its faces

    def vcycle(self):
        O().mj_rho(self.U, self.rho, self.S)
        self._vcycle_core(self.P, self.rho)

    def _vcycle_core(self, P, rho):
        """molecule.js:2879-2907: residual, restriction, 10 coarse sweeps from 0, damped prolongation."""
        S, SC = self.S, self.SC
        R = np.zeros(self.S3, np.float32)
        O().mj_residual(P, R, rho, S, self.inv_h2, np.float32(2 * np.pi))
        fc = np.zeros(SC ** 3, np.float32)
        O().mj_restrict(R, fc, S, SC)
        E = [np.zeros(SC ** 3, np.float32), np.zeros(SC ** 3, np.float32)]
        for cs in range(10):
            O().mj_coarse_smooth(E[cs % 2], E[(cs + 1) % 2], fc, SC, self.h2)
        O().mj_prolong(E[0], P, S, SC)

    def sic_pass(self):
        """molecule.js:3018-3075: per domain, solve for its own potential (4 sweeps from 0, the
        coarse correction, 4 sweeps) and subtract P_m / Z_m from Pother on the domain."""
        two_pi = np.float32(2 * np.pi)
        for m, r in enumerate(self.rows):
            Zm = np.float32(r["Z"])
            if Zm == 0:
                continue
            O().mj_rho_self(self.U, self.label, m, self.rho, self.S)
            a, b = np.zeros(self.S3, np.float32), np.zeros(self.S3, np.float32)
            for js in range(4):
                O().mj_jacobi(*((a, b) if js % 2 == 0 else (b, a)), self.rho, self.S, self.h2, two_pi)
            self._vcycle_core(a, self.rho)
            for js in range(4):
                O().mj_jacobi(*((a, b) if js % 2 == 0 else (b, a)), self.rho, self.S, self.h2, two_pi)
            O().mj_sub_self(a, self.Pother, self.label, m, Zm, self.S)

    def lobpcg_inner(self, m):
        out = np.zeros(12, np.float32)
        O().lob_inner(self.U, self.HX, self.LW, self.HW, self.LP, self.HP, self.label, m, self.S, self.h3, out)
        return out

    def lobpcg_frame(self):
        """doLOBPCGStep (molecule.js:3323-3740).  Phase 1: the Poisson solve on the current psi (the
        direct per-electron path, or 4 Jacobi sweeps and the V-cycle) and Pother (P, minus every
        domain's own potential with the self-interaction correction).  Phase 2: per domain, 10
        LOBPCG iterations (H applied to X, the Rayleigh quotient, the preconditioned residual W,
        H applied to W and P, the Ritz problem over span{X, W[, P]}, X and P updated on the
        domain).  Phase 3: normalisation, one ITP update, the level-set passes."""
        two_pi = np.float32(2 * np.pi)
        S = self.S
        poisson = self.n_electrons > 1
        if poisson and self.direct:
            for m, Pm in self.Pdirect.items():
                O().mj_rho_other(self.U, self.label, m, self.rho, S)
                scratch = np.zeros(self.S3, np.float32)
                for js in range(10):
                    O().mj_jacobi(*((Pm, scratch) if js % 2 == 0 else (scratch, Pm)), self.rho, S, self.h2, two_pi)
                O().mj_copy_for_label(Pm, self.Pother, self.label, m, S)
        elif poisson:
            O().mj_rho(self.U, self.rho, S)
            for _ in range(4):
                O().mj_jacobi(self.P, self.P2, self.rho, S, self.h2, two_pi)
                self.P, self.P2 = self.P2, self.P
            self.vcycle()
        if not poisson:
            self.Pother[:] = 0
        elif not self.direct:
            self.Pother[:] = self.P
            if self.sic:
                self.sic_pass()
        if self.frame == 0:
            self.LP[:] = 0
            self.HP[:] = 0
        at = C.addressof(self.atoms)
        for m, r in enumerate(self.rows):
            if np.float32(r["Z"]) == 0:
                continue
            for it in range(10):
                hasP = self.frame > 0 or it > 0
                O().lob_apply_h(self.U, self.HX, self.K, self.label, self.Pother, at, S, self.h, self.inv_h2)
                if it == 0 and not hasP:
                    self.LW[:] = 0
                    self.HW[:] = 0
                ip = self.lobpcg_inner(m).astype(np.float64)
                lam = np.float32(ip[1] / ip[0]) if ip[0] > 0 else np.float32(0)
                O().lob_residual(self.U, self.HX, self.LW, self.label, self.K, self.Pother, lam, m, S, self.inv_h2)
                O().lob_apply_h(self.LW, self.HW, self.K, self.label, self.Pother, at, S, self.h, self.inv_h2)
                if hasP:
                    O().lob_apply_h(self.LP, self.HP, self.K, self.label, self.Pother, at, S, self.h, self.inv_h2)
                ip2 = self.lobpcg_inner(m).astype(np.float64)
                res = np.zeros(4)
                (O().lob_ritz3 if hasP and ip2[6] > 1e-20 else O().lob_ritz2)(ip2, res)
                c = res[1:].astype(np.float32)
                O().lob_update(self.U, self.LW, self.LP, self.label, c[0], c[1], c[2], m, S)
        acc = np.zeros(self.nA, np.uint32)
        nf = np.zeros(self.nA, np.float32)
        O().mj_norms_fixed(self.U, self.label, S, self.h3, self.nA, acc, nf)
        O().mj_normalize(self.U, nf, self.label, at, S)
        O().mj_update(self.U, self.Unext, self.K, self.label, self.Pother, at, self.nA, int(self.has_bare), S, self.h,
                      self.half_d, self.dt)
        self.U, self.Unext = self.Unext, self.U
        self.frame += 1
        for _ in range(0 if self.freeze else max(1, self.spf)):
            O().mj_evolve_boundary(self.label, self.label2, self.U, self.W, S, self.dt_w, self.curv,
                                   self.lock.ctypes.data, C.addressof(self.atoms), self._splits_ptr(), self.h)
            self.label[:] = self.label2  # label2Buf -> labelBuf, all S^3 cells (molecule.js:3650)

    def step(self):
        if self.lobpcg:
            self.steps_done += 1
            self.lobpcg_frame()
            return
        self.steps_done += 1
        sf = (self.steps_done - 1) % self.spf
        poisson = self.n_electrons > 1
        if poisson and self.direct:  # molecule.js:2833-2858
            two_pi = np.float32(2 * np.pi)
            for m, Pm in self.Pdirect.items():
                O().mj_rho_other(self.U, self.label, m, self.rho, self.S)
                scratch = np.zeros(self.S3, np.float32)
                for js in range(10):
                    O().mj_jacobi(*((Pm, scratch) if js % 2 == 0 else (scratch, Pm)), self.rho, self.S, self.h2, two_pi)
                O().mj_copy_for_label(Pm, self.Pother, self.label, m, self.S)
        elif poisson:
            O().mj_rho(self.U, self.rho, self.S)
            for _ in range(self.jps):
                O().mj_jacobi(self.P, self.P2, self.rho, self.S, self.h2, np.float32(2 * np.pi))
                self.P, self.P2 = self.P2, self.P
            if sf > 0 and sf % self.vcycle_interval == 0:
                self.vcycle()
        if self.chebyshev:
            O().mj_update_cheb(self.U, self.Unext, self.K, self.label, self.Pother, C.addressof(self.atoms), self.nA,
                               self.S, self.h, self.half_d, self.dt, np.float32(self.cheb_omega_step()))
        else:
            O().mj_update(self.U, self.Unext, self.K, self.label, self.Pother, C.addressof(self.atoms), self.nA,
                          int(self.has_bare), self.S, self.h, self.half_d, self.dt)
        self.U, self.Unext = self.Unext, self.U
        if (sf + 1) % self.norm_interval == 0 or sf == self.spf - 1:
            acc = np.zeros(self.nA, np.uint32)
            nf = np.zeros(self.nA, np.float32)
            O().mj_norms_fixed(self.U, self.label, self.S, self.h3, self.nA, acc, nf)
            O().mj_normalize(self.U, nf, self.label, C.addressof(self.atoms), self.S)
        if sf == self.spf - 1:
            if not poisson:
                self.Pother[:] = 0
            elif not self.direct:  # the direct path builds Pother every step
                self.Pother[:] = self.P
            if poisson and self.sic_interval and self.frame > 0 and self.frame % self.sic_interval == 0:
                self.sic_pass()
            self.frame += 1
            for _ in range(0 if self.freeze else max(1, self.spf)):
                O().mj_evolve_boundary(self.label, self.label2, self.U, self.W, self.S, self.dt_w, self.curv,
                                      self.lock.ctypes.data, C.addressof(self.atoms), self._splits_ptr(), self.h)
                self.label[:] = self.label2  # label2Buf -> labelBuf, all S^3 cells (molecule.js:3103)
            if self.chebyshev:
                self.cheb_E = self.total_energy()

    def cheb_omega_step(self):
        """molecule.js:2924-2949 -- omega for the coming step from dv and the previous frame's E."""
        dv, E = self.dv, self.cheb_E
        dtv = dv * (self.hd * self.hd)
        dtLmax = 6.0 * dv
        dtLmin = dtv * (max(-100.0, E) if math.isfinite(E) else -10.0)
        gMax, gMin = 1 - dtLmin, 1 - dtLmax
        q = (gMax - gMin) / (gMax + gMin)
        rhoSq = q * q
        if self.cheb_state <= 1.0:
            omega, self.cheb_state = 1.0, 1.001
        elif self.cheb_state < 1.01:
            omega = 1.0 / (1.0 - rhoSq / 2.0)
            self.cheb_state = omega
        else:
            omega = 1.0 / (1.0 - rhoSq * self.cheb_state / 4.0)
            self.cheb_state = omega
        return min(1.95, max(1.0, omega))

    def total_energy(self):
        """E = E_T + E_eK + E_ee + E_KK as the page forms it (molecule.js:3124-3186): the per-H
        exclusion correction (H_RAW, :3130-3139) and the unique nuclei's softened repulsion."""
        T, EK, EE = self.energy()[:3]
        nH = sum(1 for a in self.rows if a["Z"] == 1 and (a.get("rc") or 0) == 0)
        raw = (0.5, -1.0) if self.NN in (100, 300) else (0.503, -1.028)
        T += nH * (0.5 - raw[0])
        EK += nH * (-1.0 - raw[1])
        sites = {}
        for e, a in enumerate(self.rows):
            if a["Z"] == 0 and (a.get("Z_nuc") or 0) == 0:
                continue
            key = (a["i"], a["j"], a.get("k"))
            q = (a.get("Z_nuc") or 0) or a["Z"]
            if key in sites:
                sites[key][1] += q
            else:
                sites[key] = [e, q]
        G = list(sites.values())
        ekk = 0.0
        for x in range(len(G)):
            for y in range(x + 1, len(G)):
                A, B = self.rows[G[x][0]], self.rows[G[y][0]]
                d2 = sum(((A[c] - B[c]) * self.hd) ** 2 for c in "ijk")
                ekk += G[x][1] * G[y][1] / math.sqrt(d2 + 0.04 * self.hd * self.hd)
        return T + EK + EE + ekk

    def energy(self):
        out = np.zeros(6)
        O().mj_energy(self.U, self.Pother, self.K, self.label, C.addressof(self.atoms), self.S, self.h, self.h3,
                      self.Rsing, out)
        return out


class NewMethodDriver:
    """FP64 restatement of the new flavour's schedule (Gaussian nuclei of width sigma, red-black
    multigrid V-cycle every ``poisson_interval`` steps, ITP update, FP64 normalisation to the
    domain charges after every ``norm_interval``-th update and after each update that precedes a
    V-cycle or a label pass, level-set labels every ``label_interval``).  Readouts (energy,
    forces, ``state``) first normalise psi when updates ran since the last normalisation.

    ``rows`` use the flavour's idiom: nuclei have Z_nuc > 0, domains have Z > 0 (their position
    is the seed of the initial state).  Positions are grid units (x = i*h)."""

    def __init__(self, NN, screen, rows, dv=0.2, sigma=None, poisson_interval=4, norm_interval=None, label_interval=20,
                 levels=None, pre=1, post=1, coarse_sweeps=16, boundary_speed=0.5, curv_reg=0.15, label_until=0):
        self.NN, self.S = NN, NN + 1
        self.S3 = self.S ** 3
        self.h = screen / NN
        self.sigma = sigma or self.h
        self.rows = [dict(r) for r in rows]
        self.n = len(rows)
        self.dv = dv
        self.half_dv, self.dt = 0.5 * dv, dv * self.h * self.h
        self.pi_, self.ni, self.li = poisson_interval, norm_interval or poisson_interval, label_interval
        self.age = 0  # updates since the last normalisation
        if levels is None:
            levels, nn = 1, NN
            while nn % 2 == 0 and nn // 2 >= 6:
                nn //= 2
                levels += 1
        self.levels, self.pre, self.post, self.cs = levels, pre, post, coarse_sweeps
        self.dt_w, self.curv = boundary_speed, curv_reg
        self.label_until = label_until
        self.Zdom = np.array([r.get("Z", 0.0) for r in rows], np.float64)
        self.K = np.zeros(self.S3)
        self.U = np.zeros(self.S3)
        self.U2 = np.zeros(self.S3)
        self.P = np.zeros(self.S3)
        self.label = np.zeros(self.S3, np.int32)
        self.label2 = np.zeros(self.S3, np.int32)
        self.W = np.ones(self.S3, np.float32)
        self.steps_done = 0
        self.potential()

    def nuclei(self):
        xyz = np.array([[r["i"] * self.h, r["j"] * self.h, r["k"] * self.h] for r in self.rows], np.float64)
        Z = np.array([max(r.get("Z_nuc", 0.0), 0.0) for r in self.rows], np.float64)
        return np.ascontiguousarray(xyz.reshape(-1)), Z

    def potential(self):
        xyz, Z = self.nuclei()
        O().nm_potential(self.K, xyz, Z, self.n, self.S, self.h, self.sigma)

    def set_positions(self, rows):
        self.rows = [dict(r) for r in rows]
        self.potential()

    def initialize(self, vcycles=10):
        seeds = [(q, r) for q, r in enumerate(self.rows) if r.get("Z", 0) > 0]
        hf = np.float32(self.h)
        xyz = np.array([[np.float32(r["i"] * self.h), np.float32(r["j"] * self.h), np.float32(r["k"] * self.h)]
                        for _, r in seeds], np.float32).reshape(-1)
        idx = np.array([q for q, _ in seeds], np.int32)
        O().nm_init(self.U, self.label, np.ascontiguousarray(xyz), idx, len(seeds), self.S, hf)
        self.label2[:] = self.label
        self.normalize()
        for _ in range(vcycles):
            self.vcycle()

    def domain_sums(self):
        """(sums, per domain (norm, T, V_eK, h^3 sum P rho, h^3 sum P A P)) of the current state."""
        out = np.zeros(3)
        pd = np.zeros(self.n * 5)
        O().nm_energy(self.U, self.K, self.P, self.label, self.S, self.h, out, self.n, pd)
        return out, pd.reshape(self.n, 5)

    def normalize(self):
        _, pd = self.domain_sums()
        O().nm_normalize(self.U, self.label, self.S3, self.n, self.Zdom, np.ascontiguousarray(pd[:, 0]))
        self.age = 0

    def ready(self):
        if self.age:
            self.normalize()

    def state(self):
        """(psi, label, P) as readouts see them (psi normalised)."""
        self.ready()
        return self.U, self.label, self.P

    def vcycle(self):
        O().nm_vcycle(self.P, self.U, self.S, self.h, self.levels, self.pre, self.post, self.cs)

    def step(self):
        self.steps_done += 1
        s = self.steps_done
        if s % self.pi_ == 0:
            self.vcycle()
        O().nm_update(self.U, self.U2, self.K, self.P, self.label, self.S, self.half_dv, self.dt)
        self.U, self.U2 = self.U2, self.U
        label_step = s % self.li == 0 and (self.label_until <= 0 or s <= self.label_until)
        if (s + 1) % self.ni == 0 or (s + 1) % self.pi_ == 0 or label_step:
            self.normalize()
        else:
            self.age += 1
        if label_step:
            O().nm_evolve(self.label, self.label2, self.U, self.W, self.S, float(np.float32(self.dt_w)),
                          float(np.float32(self.curv)))
            self.label, self.label2 = self.label2, self.label

    def energy(self):
        self.ready()
        out, pd = self.domain_sums()
        # kinetic and nuclear partials of the exactly normalised domains (linear in each domain's
        # density); the P-stationary Hartree energy 2 sum_d w_d h^3 sum P rho - (h^3/2pi) sum P A P
        w = np.where((self.Zdom > 0) & (pd[:, 0] > 0), self.Zdom / np.where(pd[:, 0] > 0, pd[:, 0], 1.0), 1.0)
        out = np.array([(w * pd[:, 1]).sum(), (w * pd[:, 2]).sum(),
                        2.0 * (w * pd[:, 3]).sum() - pd[:, 4].sum() / (2.0 * math.pi)])
        xyz, Z = self.nuclei()
        xyz = xyz.reshape(-1, 3)
        ekk = 0.0
        for a in range(self.n):
            for b in range(a + 1, self.n):
                if Z[a] > 0 and Z[b] > 0:
                    ekk += Z[a] * Z[b] / np.linalg.norm(xyz[a] - xyz[b])
        return {"T": out[0], "EK": out[1], "EE": out[2], "KK": ekk, "E": out.sum() + ekk, "per_domain": pd}

    def forces(self):
        self.ready()
        xyz, Z = self.nuclei()
        F = np.zeros(self.n * 3)
        O().nm_force(self.U, xyz, Z, self.n, self.S, self.h, self.sigma, F)
        return F.reshape(-1, 3)


class Shell(C.Structure):
    _fields_ = [("ne", C.c_double), ("Rmax", C.c_double), ("Zeff", C.c_double), ("split", C.c_int32),
                ("half_index", C.c_int32), ("outer_half", C.c_int32), ("fixed_w", C.c_int32)]


def shell_array(shells):
    """shells: dicts in atom.js's USER_SHELLS idiom (ne, Rmax, Zeff[, split='halfspace', halfIndex,
    outerHalf, fixedW])."""
    arr = (Shell * len(shells))()
    for q, sh in enumerate(shells):
        arr[q].ne = sh.get("ne", 1)
        arr[q].Rmax = sh.get("Rmax", 0.0) or 0.0
        arr[q].Zeff = sh["Zeff"]
        arr[q].split = 1 if sh.get("split") == "halfspace" else 0
        arr[q].half_index = int(sh.get("halfIndex", 0))
        arr[q].outer_half = int(bool(sh.get("outerHalf", False)))
        arr[q].fixed_w = int(bool(sh.get("fixedW", False)))
    return arr


class AtomShellsDriver:
    """Sequential restatement of atom.js (init :55-125, physicsStep :212-343, the multigrid
    Poisson :127-210) with JS semantics: f64 arithmetic, f32 array stores, lexicographic
    in-place loops."""

    def __init__(self, NN, screen, Z_kernel, shells, d=0.1, poisson="multigrid"):
        self.NN, self.S = NN, NN + 1
        self.S3 = self.S ** 3
        self.screen, self.Zk, self.d = float(screen), float(Z_kernel), float(d)
        self.shells = shell_array(shells)
        self.nS = len(shells)
        self.simultaneous = 1 if poisson == "simultaneous" else 0
        n = self.nS * self.S3
        self.U, self.W, self.P = (np.zeros(n, np.float32) for _ in range(3))
        self.K = np.zeros(self.S3, np.float32)

    def initialize(self):
        O().at_init(self.U, self.W, self.P, self.K, C.addressof(self.shells), self.nS, self.NN, self.screen, self.Zk)

    def step(self):
        E4 = np.zeros(4)
        ps = np.zeros(4 * self.nS)
        O().at_step(self.U, self.W, self.P, self.K, C.addressof(self.shells), self.nS, self.NN, self.screen, self.d,
                    self.simultaneous, E4, ps)
        return E4, ps.reshape(self.nS, 4)


# ---- mol_fast.js (mol_fast.js:1-1651) ----------------------------------------------------------

class MfParams(C.Structure):
    """The uniform P of mol_fast.js (writeParams, :838-874) plus its templated shader constants."""
    _fields_ = [("NN", C.c_int32), ("S", C.c_int32), ("N2", C.c_int32), ("n", C.c_int32), ("shell_mode", C.c_int32),
                ("pad0", C.c_int32), ("h", C.c_float), ("h2", C.c_float), ("inv_h", C.c_float), ("inv_h2", C.c_float),
                ("dt", C.c_float), ("half_d", C.c_float), ("h3", C.c_float), ("two_pi", C.c_float),
                ("R_out", C.c_float), ("field_x", C.c_float), ("alpha_tf", C.c_float), ("full_self", C.c_float),
                ("kc", C.c_float), ("kc_multi", C.c_float), ("beta", C.c_float), ("pad1", C.c_float),
                ("atoms", (C.c_float * 4) * 16), ("rcs", (C.c_float * 4) * 16), ("r_out", C.c_float * 16),
                ("split_type", C.c_int32 * 16), ("split_idx", C.c_int32 * 16), ("split_fix", C.c_int32 * 16),
                ("split_group", C.c_int32 * 16), ("ax", (C.c_float * 4) * 16)]


_MF_SPLIT = {"sphere": 0, "hemi": 2, "third": 3, "tetra": 4, "hemi_third": 5}


def _fixed6(v: float) -> float:
    """A number as the shader text carries it (toFixed(6)), then the literal's f32 value."""
    return float(np.float32(float(f"{v:.6f}")))


class MolFastDriver:
    """mol_fast.js restated on the CPU: the page's nucleus defaults (:28-40), the templated
    constants (:108-132), writeParams (:838-874), uploadInitialData (:941-1046), doSteps
    (:1237-1322), computeEKK (:1326-1337), computeForces (:1339-1373) and stepNuclei
    (:1375-1410), over the C restatement of the shaders (orc_mf_*)."""

    def __init__(self, nuclei, NN=200, screen=15.0, norm_targets=None, shell_mode=False, vcycle=True,
                 vcycle_interval=50, coarse_iters=10, kinetic_coeff=0.5, kc_multi=1.0, beta_pauli=0.0,
                 field_x=0.0, alpha_tf=0.0, full_self=False, r_out_release_step=None, line_j_offset=0.0,
                 dt_nuc=2.0, nuc_damping=0.9, force_scale=1.0, mass=None):
        self.nuclei = []
        for n in nuclei:
            Z = n["Z"]
            self.nuclei.append({
                "i": n["i"], "j": n["j"], "k": n["k"], "Z": Z, "rc": n.get("rc") or 0, "r_out": n.get("r_out") or 0,
                "tilt_y": n.get("tilt_y") or 0, "tilt_x": n.get("tilt_x") or 0, "hs": n.get("hs") or 0,
                "fixed": n.get("fixed") is True,
                "z_init": n["z_init"] if n.get("z_init") is not None else (Z if Z > 0 else 1),
                "split": n.get("split") or "sphere", "split_idx": n.get("split_idx") or 0,
                "split_axis": list(n.get("split_axis") or [1, 0, 0]),
                "split_fix": n["split_fix"] if n.get("split_fix") is not None else True})
        self.n = len(self.nuclei)
        self.NN, self.S = NN, NN + 1
        self.S3 = self.S ** 3
        self.N2 = round(NN / 2)
        self.hv = screen / NN
        self.h2v = self.hv * self.hv
        self.h3v = self.hv * self.hv * self.hv
        self.screen = screen
        self.tg = list(norm_targets) if norm_targets is not None else [1] * self.n
        self.vcycle, self.vi, self.ci = vcycle, vcycle_interval, coarse_iters
        self.release = r_out_release_step
        self.r_out_enforce = True
        self.dt_nuc, self.damp, self.fscale = dt_nuc, nuc_damping, force_scale
        self.mass = list(mass) if mass is not None else [max(1, a["Z"]) * 1836 for a in self.nuclei]
        self.vel = [[0.0, 0.0, 0.0] for _ in range(self.n)]
        self.force = [[0.0, 0.0, 0.0] for _ in range(self.n)]
        self.tStep = 0
        p = self.p = MfParams()
        p.NN, p.S, p.N2, p.n, p.shell_mode = NN, self.S, self.N2, self.n, 1 if shell_mode else 0
        f = lambda v: float(np.float32(v))
        p.h, p.h2, p.inv_h, p.inv_h2 = f(self.hv), f(self.h2v), f(1 / self.hv), f(1 / self.h2v)
        p.dt, p.half_d, p.h3, p.two_pi = f(0.12 * self.h2v), f(kinetic_coeff * 0.12), f(self.h3v), f(2 * math.pi)
        p.field_x, p.alpha_tf, p.full_self = f(field_x), f(alpha_tf), 1.0 if full_self else 0.0
        p.kc, p.kc_multi, p.beta = _fixed6(kinetic_coeff), _fixed6(kc_multi), _fixed6(beta_pauli)
        for a, nu in enumerate(self.nuclei):
            p.rcs[a][0], p.rcs[a][1], p.rcs[a][2], p.rcs[a][3] = nu["rc"], self.tg[a], nu["tilt_x"], nu["tilt_y"]
            p.r_out[a] = _fixed6(nu["r_out"])
            p.split_type[a] = _MF_SPLIT.get(nu["split"], 0)
            p.split_idx[a] = int(nu["split_idx"])
            p.split_fix[a] = 1 if nu["split_fix"] else 0
            v = nu["split_axis"]
            Lv = math.hypot(v[0], v[1], v[2]) or 1
            p.ax[a][0], p.ax[a][1], p.ax[a][2] = (_fixed6(v[0] / Lv), _fixed6(v[1] / Lv), _fixed6(v[2] / Lv))
            g = a
            if nu["split"] and nu["split"] != "sphere":
                for b in range(a):
                    o = self.nuclei[b]
                    if (o["split"] == nu["split"] and o["i"] == nu["i"] and o["j"] == nu["j"]
                            and o["k"] == nu["k"]):
                        g = b
                        break
            p.split_group[a] = g
        p.rcs[15][2] = line_j_offset
        self._write_atoms()
        nS = self.n * self.S3
        self.U = [np.zeros(nS, np.float32) for _ in range(2)]
        self.W = [np.zeros(nS, np.float32) for _ in range(2)]
        self.P = [np.zeros(nS, np.float32) for _ in range(2)]
        self.K = np.zeros(self.S3, np.float32)
        self.cur = 0
        self.sums = np.zeros(self.n + 6, np.float32)
        self.computeEKK()

    def _write_atoms(self):
        p = self.p
        p.R_out = 1.0 if self.r_out_enforce else 0.0
        for a, nu in enumerate(self.nuclei):
            p.atoms[a][0], p.atoms[a][1], p.atoms[a][2], p.atoms[a][3] = nu["i"], nu["j"], nu["k"], nu["Z"]

    @property
    def pp(self):
        return C.addressof(self.p)

    def initialize(self):
        rec = np.zeros((self.n, 16))
        for a, nu in enumerate(self.nuclei):
            ax = nu["split_axis"]
            rec[a, :14] = [nu["i"], nu["j"], nu["k"], nu["Z"], nu["rc"], nu["r_out"], nu["hs"], nu["z_init"],
                           self.tg[a], _MF_SPLIT.get(nu["split"], 0), nu["split_idx"], ax[0], ax[1], ax[2]]
        O().mf_init(self.NN, self.screen, self.n, np.ascontiguousarray(rec.reshape(-1)), self.K, self.U[0], self.W[0],
                    self.P[0])
        for X in (self.U, self.W, self.P):
            X[1][:] = X[0]
        self.cur = 0

    def computeEKK(self):
        E = 0.0
        nu = self.nuclei
        for a in range(self.n):
            for b in range(a + 1, self.n):
                dx, dy, dz = ((nu[a][c] - nu[b][c]) * self.hv for c in "ijk")
                r = math.sqrt(dx * dx + dy * dy + dz * dz)
                if r > 0:
                    E += nu[a]["Z"] * nu[b]["Z"] / r
        self.E_KK = E

    def do_steps(self, n):
        if self.release is not None and self.r_out_enforce and self.tStep >= self.release:
            self.r_out_enforce = False
            self._write_atoms()
        o = O()
        for s in range(n):
            c, nx = self.cur, 1 - self.cur
            o.mf_update(self.pp, self.U[c], self.W[c], self.P[c], self.K, self.U[nx], self.W[nx], self.P[nx])
            if (s + 1) % 20 == 0 or s == n - 1:
                o.mf_reduce(self.pp, self.U[nx], self.W[nx], self.P[nx], self.K, self.sums)
                o.mf_normalize(self.pp, self.U[nx], self.sums)
            if self.vcycle and (s + 1) % self.vi == 0:
                for m in range(self.n):
                    o.mf_vcycle(self.pp, self.U[nx], self.P[nx], m, self.ci)
            self.cur = nx
        ne, sm = self.n, self.sums
        self.E_T, self.E_eK, self.E_ee = float(sm[ne]), float(sm[ne + 1]), float(sm[ne + 2])
        self.E = self.E_T + self.E_eK + self.E_ee + self.E_KK
        dn = [0.0, 0.0, 0.0]
        for a in self.nuclei:
            dn[0] += a["Z"] * (a["i"] - self.N2) * self.hv
            dn[1] += a["Z"] * (a["j"] - self.N2) * self.hv
            dn[2] += a["Z"] * (a["k"] - self.N2) * self.hv
        self.dipole = [dn[0] + float(sm[ne + 3]), dn[1] + float(sm[ne + 4]), dn[2] + float(sm[ne + 5])]
        self.tStep += n

    def compute_forces(self):
        fd = np.zeros(3 * self.n, np.float32)
        O().mf_force(self.pp, self.P[self.cur], fd)
        nu = self.nuclei
        for a in range(self.n):
            f = [float(fd[3 * a]), float(fd[3 * a + 1]), float(fd[3 * a + 2])]
            for b in range(self.n):
                if b == a:
                    continue
                dx, dy, dz = ((nu[a][c] - nu[b][c]) * self.hv for c in "ijk")
                r2 = dx * dx + dy * dy + dz * dz + self.h2v
                inv_r3 = 1 / (r2 * math.sqrt(r2))
                pref = nu[a]["Z"] * nu[b]["Z"] * inv_r3
                f[0] += pref * dx
                f[1] += pref * dy
                f[2] += pref * dz
            self.force[a] = f
        return fd

    def step_nuclei(self):
        moved = False
        for a, nu in enumerate(self.nuclei):
            if nu["Z"] <= 0 or nu["fixed"]:
                continue
            v = self.vel[a]
            for d in range(3):
                v[d] = self.damp * (v[d] + self.dt_nuc * self.fscale * self.force[a][d] / self.mass[a])
            di, dj, dk = (v[0] * self.dt_nuc) / self.hv, (v[1] * self.dt_nuc) / self.hv, (v[2] * self.dt_nuc) / self.hv
            if abs(di) > 0.0001 or abs(dj) > 0.0001 or abs(dk) > 0.0001:
                nu["i"] += di
                nu["j"] += dj
                nu["k"] += dk
                moved = True
        if moved:
            self._write_atoms()
            self.computeEKK()
            O().mf_recompute_k(self.pp, self.K)
        return moved

    def extract(self):
        out = np.zeros(3 * self.n * self.S * self.S, np.float32)
        c = self.cur
        O().mf_extract(self.pp, self.U[c], self.W[c], self.P[c], out)
        return out

    def fields(self, m):
        c, S3 = self.cur, self.S3
        return {"U": self.U[c][m * S3:(m + 1) * S3], "W": self.W[c][m * S3:(m + 1) * S3],
                "P": self.P[c][m * S3:(m + 1) * S3]}


# ---- realqm_rb.js (realqm_rb.js:1-1222) ---------------------------------------------------------

class RbParams(C.Structure):
    _fields_ = [("NN", C.c_int32), ("S", C.c_int32), ("N2", C.c_int32), ("n", C.c_int32), ("h", C.c_float),
                ("h2", C.c_float), ("inv_h", C.c_float), ("inv_h2", C.c_float), ("dt", C.c_float),
                ("half_d", C.c_float), ("two_pi", C.c_float), ("h3", C.c_float), ("tgt", C.c_float * 16)]


class RealqmRbDriver:
    """realqm_rb.js restated on the CPU: the page constants (:8-35), electronNucleus (:73-82),
    runInitKernels and the r_c masks (:720-801, :519-544, :615-644), doSteps (:891-965) with the
    reference's sequential per-electron passes, computeEnergy (:982-1045), extractSlice."""

    def __init__(self, nuclei, NN=100, screen=8.0, norm_targets=None):
        self.nuclei = [dict(n, ne=1 if n.get("ne") is None else n["ne"], rc=n.get("rc") or 0) for n in nuclei]
        self.enuc = [a for a, nu in enumerate(self.nuclei) for _ in range(int(nu["ne"]))]
        self.n = len(self.enuc)
        self.NN, self.S = NN, NN + 1
        self.S3 = self.S ** 3
        self.h = screen / NN
        self.h2, self.h3 = self.h * self.h, self.h * self.h * self.h
        p = self.p = RbParams()
        f = lambda v: float(np.float32(v))
        p.NN, p.S, p.N2, p.n = NN, self.S, NN // 2, self.n
        p.h, p.h2, p.inv_h, p.inv_h2 = f(self.h), f(self.h2), f(1 / self.h), f(1 / self.h2)
        p.dt, p.half_d, p.two_pi, p.h3 = f(0.1 * self.h2), f(0.5 * 0.1), f(2 * math.pi), f(self.h3)
        for m in range(self.n):
            p.tgt[m] = norm_targets[m] if norm_targets is not None else self.nuclei[self.enuc[m]]["ne"]
        nS = self.n * self.S3
        self.U, self.W, self.P = (np.zeros(nS, np.float32) for _ in range(3))
        self.K = np.zeros(self.S3, np.float32)
        self.mask = np.ones(nS, np.float32)
        self.rho = np.zeros(self.S3, np.float32)
        self.unear = np.zeros(nS, np.float32)
        self.norms = np.zeros(self.n, np.float32)

    @property
    def pp(self):
        return C.addressof(self.p)

    def initialize(self):
        nuc = np.zeros((len(self.nuclei), 8), np.float32)
        for a, nu in enumerate(self.nuclei):
            nuc[a, :6] = [nu["i"], nu["j"], nu["k"], nu["Z"], nu["rc"], nu["ne"]]
        O().rb_init(self.pp, len(self.nuclei), np.ascontiguousarray(nuc.reshape(-1)),
                    np.array(self.enuc, np.int32), self.K, self.U, self.W, self.P)
        S, S2, h = self.S, self.S * self.S, self.h
        for m in range(self.n):  # the r_c exclusion masks, in JS numbers
            nu = self.nuclei[self.enuc[m]]
            rc = nu.get("rc_excl") or 0
            if not rc > 0 or any(float(nu[c]) != math.floor(nu[c]) for c in "ijk"):
                continue
            rcc = math.ceil(rc / h) + 1
            for di in range(-rcc, rcc + 1):
                for dj in range(-rcc, rcc + 1):
                    for dk in range(-rcc, rcc + 1):
                        gi, gj, gk = int(nu["i"]) + di, int(nu["j"]) + dj, int(nu["k"]) + dk
                        if gi < 0 or gi >= S or gj < 0 or gj >= S or gk < 0 or gk >= S:
                            continue
                        r2 = (di * h) * (di * h) + (dj * h) * (dj * h) + (dk * h) * (dk * h)
                        if r2 < rc * rc:
                            idx = m * self.S3 + gi * S2 + gj * S + gk
                            self.mask[idx] = 0.0
                            self.U[idx] = 0.0
                            self.W[idx] = 0.0

    def do_steps(self, n):
        o = O()
        for s in range(n):
            o.rb_rho_nearest(self.pp, self.U, self.rho, self.unear)
            for color in (0, 1):
                for m in range(self.n):
                    o.rb_wu(self.pp, m, color, self.U, self.W, self.unear, self.K, self.P, self.mask)
                for m in range(self.n):
                    o.rb_p(self.pp, m, color, self.P, self.U, self.rho)
            if s % 5 == 0:
                for m in range(self.n):
                    self.norms[m] = o.rb_normalize(self.pp, m, self.U)

    def energy(self):
        out = np.zeros(3)
        O().rb_energy(self.pp, self.U, self.W, self.P, self.K, self.h, self.h3, out)
        return out

    def slice(self):
        out = np.zeros(self.S * self.S * (3 * self.n + 1), np.float32)
        O().rb_slice(self.pp, self.U, self.W, self.P, self.K, out)
        return out

    def fields(self, m):
        S3 = self.S3
        return {"U": self.U[m * S3:(m + 1) * S3], "W": self.W[m * S3:(m + 1) * S3], "P": self.P[m * S3:(m + 1) * S3]}
