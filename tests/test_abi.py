"""The C-ABI library loads and exports every entry point include/rq.h declares (CPU only)."""
import ctypes
import os
import re

import pytest

from realmolecule_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            with open(os.path.join(inc, fn)) as f:
                names |= set(re.findall(r"^RQ_API\s+[^;(]*?\b(rq_\w+)\s*\(", f.read(), flags=re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "rq_create" in names and "rq_step" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared_symbols()) <= set(_lib.SIGNATURES), set(declared_symbols()) - set(_lib.SIGNATURES)


def test_status_strings():
    lib = _lib.load()
    assert lib.rq_status_string(0) == b"ok"
    assert lib.rq_status_string(-1) == b"invalid argument"
    assert lib.rq_status_string(-7) == b"no CUDA device"
    assert lib.rq_status_string(5) == b"unknown status"


def test_create_rejects_bad_config_without_touching_a_device():
    lib = _lib.load()
    cfg = _lib.Config()
    cfg.NN = 33  # odd NN: multigrid needs an even NN (molecule.js:155)
    cfg.screen = 8.0
    atoms = (_lib.Atom * 1)()
    atoms[0].i = atoms[0].j = atoms[0].k = 16
    atoms[0].Z = 1
    h = ctypes.c_void_p()
    assert lib.rq_create(ctypes.byref(cfg), atoms, 1, ctypes.byref(h)) == _lib.RQ_EINVAL
    cfg.NN = 32
    cfg.precision = 1  # FP64 only exists for the new flavour
    cfg.flavor = 1
    assert lib.rq_create(ctypes.byref(cfg), atoms, 1, ctypes.byref(h)) == _lib.RQ_ENOTSUP
    assert lib.rq_create(ctypes.byref(cfg), atoms, 0, ctypes.byref(h)) == _lib.RQ_EINVAL
    cfg.precision = 0
    cfg.flavor = 1  # solver.py
    cfg.lobpcg = 1  # LOBPCG frames are molecule.js's
    assert lib.rq_create(ctypes.byref(cfg), atoms, 1, ctypes.byref(h)) == _lib.RQ_ENOTSUP
    cfg.flavor = 0  # molecule.js
    cfg.chebyshev = 1  # the page runs one of the two alternatives at a time
    assert lib.rq_create(ctypes.byref(cfg), atoms, 1, ctypes.byref(h)) == _lib.RQ_EINVAL


def test_kernel_entry_points_validate_arguments():
    lib = _lib.load()
    assert lib.rq_kernel_update_sp(None, None, None, None, None, 17, 0.06, 0.01, None) == _lib.RQ_EINVAL
    assert lib.rq_kernel_labels_sp(None, None, None, 1, 17, 0.25, 0.0625, None) == _lib.RQ_EINVAL


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from realmolecule_b200 import Context
    with pytest.raises(_lib.RqError) as e:
        Context(16, 4.0, [{"i": 8, "j": 8, "k": 8, "Z": 1}])
    assert e.value.status == _lib.RQ_ENODEV
