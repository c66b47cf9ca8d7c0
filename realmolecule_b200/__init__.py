"""realmolecule_b200 -- a B200-native RealQM real-space solver step.

The solver step (fused ITP update with FP64 per-domain sums, the integer label /
level-set update, the Poisson solve and the atom-centre force gather) runs as
hand-written sm_100a CUDA kernels in ``librq.so`` behind the C ABI of
``include/rq.h``.  This package is the Python host over that ABI:

* ``RealQMSolver``  -- drop-in for cloud/solver.py's class (same config, run(), snapshots);
* ``Context``       -- one librq context (any flavour / precision) with numpy I/O;
* ``build``         -- compile librq.so in-tree for sm_100a.
"""
from . import _lib  # noqa: F401
from .context import Context  # noqa: F401
from .solver import RealQMSolver  # noqa: F401

__all__ = ["Context", "RealQMSolver"]
