"""ctypes binding of librq (include/rq.h).

The library is built in-tree by ``python -m realmolecule_b200.build`` and loaded from the
package directory.  There is no fallback: if librq.so is missing or no CUDA device is
visible, the calls fail with an exception naming the reason.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "librq.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "rq.h")

RQ_OK, RQ_EINVAL, RQ_ENOMEM, RQ_ECUDA, RQ_ENONFINITE, RQ_ETIMEOUT, RQ_ENOTSUP, RQ_ENODEV = 0, -1, -2, -3, -4, -5, -6, -7
FLAVOR_MOLECULE_JS, FLAVOR_SOLVER_PY, FLAVOR_NEW = 0, 1, 2
PREC_MIXED, PREC_FP64 = 0, 1
FORCE_HF, FORCE_GRADP, FORCE_ADJOINT = 0, 1, 2
E_TOTAL, E_T, E_EK, E_EE, E_KK, E_DIPX, E_DIPY, E_DIPZ = range(8)
ENERGY_LEN, DOMAIN_LEN = 8, 5
NOALLOC_MAX_DOMAINS = 16384


class RqError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: status {status} ({status_string(status)}){': ' + detail if detail else ''}")


class ShellsConfig(C.Structure):
    _fields_ = [("NN", C.c_int32), ("poisson", C.c_int32), ("screen", C.c_double), ("Z_kernel", C.c_double),
                ("d", C.c_double), ("reserved", C.c_int32 * 4)]


class Shell(C.Structure):
    _fields_ = [("ne", C.c_double), ("Rmax", C.c_double), ("Zeff", C.c_double), ("split", C.c_int32),
                ("half_index", C.c_int32), ("outer_half", C.c_int32), ("fixed_w", C.c_int32)]


class MfConfig(C.Structure):
    _fields_ = [("NN", C.c_int32), ("shell_mode", C.c_int32), ("vcycle", C.c_int32), ("vcycle_interval", C.c_int32),
                ("coarse_iters", C.c_int32), ("r_out_release_step", C.c_int32), ("full_self", C.c_int32),
                ("reserved0", C.c_int32), ("screen", C.c_double), ("kinetic_coeff", C.c_double),
                ("kc_multi", C.c_double), ("beta_pauli", C.c_double), ("field_x", C.c_double),
                ("alpha_tf", C.c_double), ("line_j_offset", C.c_double), ("reserved", C.c_int32 * 8)]


class MfNucleus(C.Structure):
    _fields_ = [("i", C.c_double), ("j", C.c_double), ("k", C.c_double), ("Z", C.c_double), ("rc", C.c_double),
                ("r_out", C.c_double), ("tilt_y", C.c_double), ("tilt_x", C.c_double), ("hs", C.c_double),
                ("z_init", C.c_double), ("norm_target", C.c_double), ("split_axis", C.c_double * 3),
                ("split", C.c_int32), ("split_idx", C.c_int32), ("split_fix", C.c_int32), ("reserved", C.c_int32)]


class RbConfig(C.Structure):
    _fields_ = [("NN", C.c_int32), ("reserved0", C.c_int32), ("screen", C.c_double), ("reserved", C.c_int32 * 8)]


class RbNucleus(C.Structure):
    _fields_ = [("i", C.c_double), ("j", C.c_double), ("k", C.c_double), ("Z", C.c_double), ("rc", C.c_double),
                ("rc_excl", C.c_double), ("ne", C.c_int32), ("reserved", C.c_int32)]


class Config(C.Structure):
    _fields_ = [("NN", C.c_int32), ("flavor", C.c_int32), ("precision", C.c_int32), ("norm_interval", C.c_int32),
                ("screen", C.c_double), ("dv", C.c_double), ("poisson_interval", C.c_int32),
                ("label_interval", C.c_int32), ("jacobi_per_step", C.c_int32), ("steps_per_frame", C.c_int32),
                ("vcycle_interval", C.c_int32), ("mg_levels", C.c_int32), ("mg_pre", C.c_int32),
                ("mg_post", C.c_int32), ("mg_coarse_sweeps", C.c_int32), ("sic", C.c_int32),
                ("boundary_speed", C.c_double), ("curv_reg", C.c_double), ("sigma", C.c_double),
                ("label_until", C.c_int32), ("chebyshev", C.c_int32), ("lobpcg", C.c_int32),
                ("converge_checks", C.c_int32), ("fp32_rounding", C.c_int32), ("nuclear_sum", C.c_int32),
                ("batch_persistent", C.c_int32), ("batch_tile", C.c_int32)]


class TuneReport(C.Structure):
    _fields_ = [("n_tile", C.c_int32), ("tile", C.c_int32 * 12), ("persistent", C.c_int32 * 12),
                ("ms_per_step", C.c_double * 12), ("n_smooth", C.c_int32), ("pre", C.c_int32 * 8),
                ("post", C.c_int32 * 8), ("coarse_sweeps", C.c_int32 * 8), ("rho", C.c_double * 8),
                ("ms_per_cycle", C.c_double * 8), ("best_tile", C.c_int32), ("best_smooth", C.c_int32),
                ("reserved", C.c_int32 * 6)]


class Split(C.Structure):
    _fields_ = [("type", C.c_int32), ("idx", C.c_int32), ("axis", C.c_double * 3), ("rot", C.c_double)]


class Atom(C.Structure):
    _fields_ = [("i", C.c_double), ("j", C.c_double), ("k", C.c_double), ("Z", C.c_double), ("Z_nuc", C.c_double),
                ("rc", C.c_double), ("init_zeff", C.c_double), ("init_rcut", C.c_double)]


class Info(C.Structure):
    _fields_ = [("NN", C.c_int32), ("S", C.c_int32), ("n_atoms", C.c_int32), ("flavor", C.c_int32),
                ("precision", C.c_int32), ("steps_done", C.c_int32), ("mg_levels", C.c_int32), ("_pad", C.c_int32),
                ("h", C.c_double), ("dv", C.c_double), ("dt", C.c_double), ("sigma", C.c_double),
                ("S3", C.c_int64), ("psi", C.c_void_p), ("label", C.c_void_p), ("K", C.c_void_p),
                ("P", C.c_void_p), ("W", C.c_void_p), ("kernel_launches", C.c_int64)]


KC_UPDATE, KC_POISSON, KC_LABELS, KC_NORMALIZE, KC_ENERGY, KC_FORCES, KC_MG, KC_OTHER = range(8)
KC_NAMES = ["update", "poisson", "labels", "normalize", "energy", "forces", "multigrid", "other"]


class Profile(C.Structure):
    _fields_ = [("launches", C.c_int64 * 8), ("ms", C.c_double * 8), ("bytes", C.c_double * 8)]


_V, _P, _I, _F, _D = C.c_void_p, C.c_void_p, C.c_int32, C.c_float, C.c_double
_DP = C.POINTER(C.c_double)

# name -> (restype, argtypes); every symbol include/rq.h declares
SIGNATURES = {
    "rq_create": (C.c_int, [C.POINTER(Config), C.POINTER(Atom), _I, C.POINTER(C.c_void_p)]),
    "rq_destroy": (None, [_V]),
    "rq_set_stream": (C.c_int, [_V, _V]),
    "rq_get_info": (C.c_int, [_V, C.POINTER(Info)]),
    "rq_last_error": (C.c_char_p, [_V]),
    "rq_status_string": (C.c_char_p, [C.c_int]),
    "rq_initialize": (C.c_int, [_V]),
    "rq_set_atoms": (C.c_int, [_V, C.POINTER(Atom), _I]),
    "rq_set_external_potential": (C.c_int, [_V, _P]),
    "rq_upload_state": (C.c_int, [_V, _P, _P, _P, _P]),
    "rq_download_state": (C.c_int, [_V, _P, _P, _P, _P]),
    "rq_upload_state_f64": (C.c_int, [_V, _P, _P]),
    "rq_download_state_f64": (C.c_int, [_V, _P, _P, _P]),
    "rq_download_K": (C.c_int, [_V, _P]),
    "rq_step": (C.c_int, [_V, _I]),
    "rq_energy": (C.c_int, [_V, _P, _P]),
    "rq_forces": (C.c_int, [_V, _I, _P]),
    "rq_nuclear_terms": (C.c_int, [_V, _DP, _P]),
    "rq_promote": (C.c_int, [_V]),
    "rq_set_adjoint_window": (C.c_int, [_V, _I]),
    "rq_adjoint": (C.c_int, [_V, _P, _P]),
    "rq_extract": (C.c_int, [_V, _I, _P]),
    "rq_solve": (C.c_int, [_V, _D, _I, _I, C.POINTER(C.c_int32), _DP]),
    "rq_synchronize": (C.c_int, [_V]),
    "rq_profile_begin": (C.c_int, [_V]),
    "rq_profile_end": (C.c_int, [_V, C.POINTER(Profile)]),
    "rq_batch_create": (C.c_int, [C.POINTER(Config), C.POINTER(Atom), C.POINTER(C.c_int32), _I,
                                  C.POINTER(C.c_void_p)]),
    "rq_batch_destroy": (None, [_V]),
    "rq_batch_last_error": (C.c_char_p, [_V]),
    "rq_batch_set_stream": (C.c_int, [_V, _V]),
    "rq_batch_initialize": (C.c_int, [_V]),
    "rq_batch_step": (C.c_int, [_V, _I]),
    "rq_batch_energy": (C.c_int, [_V, _P]),
    "rq_batch_forces": (C.c_int, [_V, _P]),
    "rq_batch_solve": (C.c_int, [_V, _D, _I, _I, _P, _P]),
    "rq_batch_info": (C.c_int, [_V, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                C.POINTER(C.c_int64)]),
    "rq_batch_synchronize": (C.c_int, [_V]),
    "rq_batch_set_wait": (C.c_int, [_V, C.c_int64, _I]),
    "rq_batch_autotune": (C.c_int, [_V, _P]),
    "rq_shells_create": (C.c_int, [_P, _P, _I, _P]),
    "rq_shells_destroy": (None, [_V]),
    "rq_shells_last_error": (C.c_char_p, [_V]),
    "rq_shells_step": (C.c_int, [_V, _I, _P, _P]),
    "rq_shells_download": (C.c_int, [_V, _I, _P, _P, _P]),
    "rq_shells_upload": (C.c_int, [_V, _I, _P, _P, _P]),
    "rq_shells_info": (C.c_int, [_V, _P]),
    "rq_mf_create": (C.c_int, [_P, _P, _I, _P]),
    "rq_mf_destroy": (None, [_V]),
    "rq_mf_last_error": (C.c_char_p, [_V]),
    "rq_mf_step": (C.c_int, [_V, _I, _P]),
    "rq_mf_forces": (C.c_int, [_V, _P]),
    "rq_mf_set_positions": (C.c_int, [_V, _P]),
    "rq_mf_extract": (C.c_int, [_V, _P]),
    "rq_mf_download": (C.c_int, [_V, _I, _P, _P, _P]),
    "rq_mf_upload": (C.c_int, [_V, _I, _P, _P, _P]),
    "rq_mf_download_K": (C.c_int, [_V, _P]),
    "rq_mf_info": (C.c_int, [_V, _P, _P]),
    "rq_rb_create": (C.c_int, [_P, _P, _I, _P, _P]),
    "rq_rb_destroy": (None, [_V]),
    "rq_rb_last_error": (C.c_char_p, [_V]),
    "rq_rb_step": (C.c_int, [_V, _I]),
    "rq_rb_energy": (C.c_int, [_V, _P]),
    "rq_rb_slice": (C.c_int, [_V, _P]),
    "rq_rb_download": (C.c_int, [_V, _I, _P, _P, _P]),
    "rq_rb_upload": (C.c_int, [_V, _I, _P, _P, _P]),
    "rq_rb_download_K": (C.c_int, [_V, _P]),
    "rq_rb_info": (C.c_int, [_V, _P, _P]),
    "rq_set_locked_groups": (C.c_int, [_V, _I, _P, _P]),
    "rq_set_splits": (C.c_int, [_V, _P]),
    "rq_restart": (C.c_int, [_V]),
    "rq_set_freeze_boundary": (C.c_int, [_V, _I]),
    "rq_set_init_positions": (C.c_int, [_V, _P, _P, _I]),
    "rq_kernel_update_sp": (C.c_int, [_P, _P, _P, _P, _P, _I, _F, _F, _V]),
    "rq_kernel_jacobi_sp": (C.c_int, [_P, _P, _P, _I, _F, _F, _V]),
    "rq_kernel_labels_sp": (C.c_int, [_P, _P, _P, _I, _I, _F, _F, _V]),
    "rq_kernel_init_sp": (C.c_int, [_P, _P, _P, _P, _P, _I, _I, _F, _F, _V]),
    "rq_kernel_recompute_k_sp": (C.c_int, [_P, _P, _I, _I, _F, _F, _V]),
    "rq_kernel_normalize_sp": (C.c_int, [_P, _P, _P, _I, _I, _F, _P, _V]),
    "rq_kernel_normalize_sp_noalloc": (C.c_int, [_P, _P, _P, _I, _I, _F, _V]),
    "rq_kernel_energy_sp": (C.c_int, [_P, _P, _P, _P, _I, _I, _F, _F, _P, _V]),
    "rq_kernel_forces_hf_sp": (C.c_int, [_P, _P, _I, _I, _F, _F, _F, _P, _V]),
}

_lib = None


def load():
    """Load librq.so (built in-tree).  Raises if it is missing -- there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"librq.so not built at {LIB_PATH}; run `python -m realmolecule_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def status_string(status: int) -> str:
    try:
        return load().rq_status_string(status).decode()
    except Exception:  # pragma: no cover - only when the library itself is missing
        return "?"


def check(status: int, where: str, ctx=None):
    if status != RQ_OK:
        detail = ""
        if ctx is not None:
            try:
                detail = load().rq_last_error(ctx).decode()
            except Exception:
                pass
        raise RqError(status, where, detail)
    return status
