"""numpy-backed stand-in for the few cupy calls cloud/solver.py makes (TEST INFRASTRUCTURE).

Lets the untouched reference ``RealQMSolver`` (cloud/solver.py:318-638) run on the host
of THIS container so that tests/golden/make_golden.py can record its outputs.  Each
``RawKernel`` is dispatched to the reference's own kernel text compiled for the host
(oracle/_ref/libsolverpy_ref.so); ``computeEnergy`` (shared memory + __syncthreads) is
dispatched to its restatement in oracle/rq_oracle.c.
"""
import os
import sys

import numpy as np

from . import cuda  # noqa: F401

float32 = np.float32
int32 = np.int32

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(_HERE)))  # oracle/
import oracle as _oracle  # noqa: E402

SERIAL = False  # run kernels single-threaded in index order (deterministic in-place races)


class ndarray(np.ndarray):
    def get(self):
        return np.asarray(self).copy()


def zeros(n, dtype=np.float32):
    return np.zeros(n, dtype).view(ndarray)


def asarray(a):
    return np.ascontiguousarray(a).view(ndarray)


_REF = None


class RawKernel:
    def __init__(self, src, name):
        self.name = name

    def __call__(self, grid, block, args, shared_mem=0):
        global _REF
        if self.name == "computeEnergy":
            U, K, P, label, out, S, h, h3 = args
            tmp = np.zeros(3, np.float32)
            _oracle.O().sp_energy_blocktree(np.asarray(U), np.asarray(K), np.asarray(P), np.asarray(label), tmp,
                                            int(S), float(h), float(h3), int(block[0]))
            out += tmp
            return
        if _REF is None:
            _REF = _oracle.RefKernels()
        _REF.launch(self.name, grid[0], block[0], [np.asarray(a) if isinstance(a, np.ndarray) else a for a in args],
                    serial=SERIAL)
