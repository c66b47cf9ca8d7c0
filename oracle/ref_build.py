"""Build recipe: compile the reference's cloud/solver.py kernels for the host CPU.

TEST INFRASTRUCTURE ONLY (oracle + CPU baseline).  The product never imports this.

The reference keeps its nine CUDA-C kernels as string literals handed to
``cupy.RawKernel`` (cloud/solver.py:16-315).  This recipe reads those strings from
the reference tree where they lie, writes them unchanged into the git-ignored
``oracle/_ref/`` folder, appends one OpenMP launcher per kernel and compiles the
result with g++ (no FMA contraction, no fast-math) into
``oracle/_ref/libsolverpy_ref.so``.  Kernels that rely on ``__syncthreads`` and
dynamic shared memory (only ``computeEnergy``, cloud/solver.py:227-280) are not
compiled; the oracle restates that one (oracle/rq_oracle.c).

The built .so travels with the repository snapshot to machines without the
reference tree; nothing here runs there.

Usage:  python oracle/ref_build.py [--reference DIR] [--force]

The reference tree is DIR, else the environment variable REALQM_REFERENCE_DIR, else
/root/reference (where the build container mounts it).
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libsolverpy_ref.so")
DEFAULT_REFERENCE = os.environ.get("REALQM_REFERENCE_DIR", "/root/reference")

_KERNEL_RE = re.compile(r"cp\.RawKernel\(r'''(.*?)''',\s*'(\w+)'\)", re.S)
_SIG_RE = re.compile(r"void\s+(\w+)\s*\(([^)]*)\)", re.S)


def extract_kernels(src: str):
    """Return [(name, source, [(ctype, pname), ...], uses_sync)] from solver.py text."""
    out = []
    for body, name in _KERNEL_RE.findall(src):
        m = _SIG_RE.search(body)
        if not m or m.group(1) != name:
            raise RuntimeError(f"cannot parse signature of kernel {name}")
        params = []
        for p in m.group(2).split(","):
            p = " ".join(p.split())
            pm = re.match(r"(.*?)(\w+)$", p)
            params.append((pm.group(1).strip(), pm.group(2)))
        out.append((name, body, params, "__syncthreads" in body))
    return out


def _launcher(name, params):
    decl = ", ".join(f"{t} {n}" for t, n in params)
    args = ", ".join(n for _, n in params)
    return f"""
extern "C" void rqref_launch_{name}(int grid_x, int block_x{', ' + decl if decl else ''}) {{
#pragma omp parallel for schedule(static)
  for (int b = 0; b < grid_x; ++b) {{
    blockIdx.x = (unsigned)b; blockDim.x = (unsigned)block_x; gridDim.x = (unsigned)grid_x;
    for (int t = 0; t < block_x; ++t) {{ threadIdx.x = (unsigned)t; {name}({args}); }}
  }}
}}
extern "C" void rqref_launch_serial_{name}(int grid_x, int block_x{', ' + decl if decl else ''}) {{
  for (int b = 0; b < grid_x; ++b) {{
    blockIdx.x = (unsigned)b; blockDim.x = (unsigned)block_x; gridDim.x = (unsigned)grid_x;
    for (int t = 0; t < block_x; ++t) {{ threadIdx.x = (unsigned)t; {name}({args}); }}
  }}
}}
"""


def build(reference: str = DEFAULT_REFERENCE, force: bool = False, quiet: bool = False) -> str:
    src_path = os.path.join(reference, "cloud", "solver.py")
    if not os.path.exists(src_path):
        if os.path.exists(LIB):
            return LIB
        raise FileNotFoundError(f"reference solver not found at {src_path} and no prebuilt {LIB}")
    os.makedirs(OUT_DIR, exist_ok=True)
    with open(src_path) as f:
        src = f.read()
    kernels = extract_kernels(src)
    cpp = os.path.join(OUT_DIR, "solverpy_kernels.cpp")
    parts = ["// generated by oracle/ref_build.py from cloud/solver.py; do not commit\n"]
    names = []
    for name, body, params, uses_sync in kernels:
        if uses_sync:
            continue
        parts.append(body)
        parts.append(_launcher(name, params))
        names.append(name)
    text = "\n".join(parts)
    if (not force and os.path.exists(LIB) and os.path.exists(cpp)
            and open(cpp).read() == text and os.path.getmtime(LIB) >= os.path.getmtime(cpp)):
        return LIB
    with open(cpp, "w") as f:
        f.write(text)
    cmd = ["g++", "-O3", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
           "-include", os.path.join(HERE, "cuda_host_shim.h"), "-x", "c++", cpp, "-o", LIB]
    if not quiet:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    with open(os.path.join(OUT_DIR, "kernels.txt"), "w") as f:
        f.write("\n".join(names) + "\n")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.reference, a.force))
    sys.exit(0)
