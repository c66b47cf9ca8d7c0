"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in a container that has the reference tree (--reference, else REALQM_REFERENCE_DIR, else
/root/reference):

    python tests/golden/make_golden.py [--reference DIR]

What it records (all small, committed):

* ``solverpy_kernels_nn16.npz`` -- inputs and outputs of each cloud/solver.py kernel
  (compiled for the host from the reference's own kernel text by oracle/ref_build.py),
  run once on a seeded state of a 17^3 grid.  Labels from ``boundaryEvolve`` are the
  serial in-place result (the reference kernel writes labels in place).
* ``solverpy_run_h2o_nn32.json`` -- energies from the UNMODIFIED reference
  ``RealQMSolver`` (cloud/solver.py:318-638) driven through a numpy stand-in for cupy
  (oracle/fake_cupy), kernels run serially, for a 3-domain valence H2O on 33^3, 200 steps.
* ``hairpin_config.json`` -- the atom list built by ``build_hairpin_config``
  (cloud/run_hairpin.py:21-182), 267 atoms on NN=300.
* ``hairpin_golden.json`` -- the energy components per snapshot and the final nuclear
  positions recorded by the reference in cloud/hairpin_results.json (A100 run).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle", "fake_cupy"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def seeded_state(NN: int, n_atoms: int, seed: int):
    """A physically shaped random state: atoms inside the box, psi > 0 with
    exponential tails, labels = nearest atom, P a smooth positive field."""
    rng = np.random.default_rng(seed)
    S = NN + 1
    pos = rng.uniform(4, NN - 4, size=(n_atoms, 3)).astype(np.float32)
    Z = rng.integers(1, 4, size=n_atoms).astype(np.float32)
    rc = np.where(rng.random(n_atoms) < 0.3, 0.4, 0.0).astype(np.float32)
    g = np.arange(S, dtype=np.float32)
    I, J, K = np.meshgrid(g, g, g, indexing="ij")
    d2 = np.stack([(I - p[0]) ** 2 + (J - p[1]) ** 2 + (K - p[2]) ** 2 for p in pos])
    label = np.argmin(d2, axis=0).astype(np.int32)
    U = (np.exp(-0.3 * np.sqrt(d2.min(axis=0))) * (1 + 0.1 * rng.random(d2.shape[1:]))).astype(np.float32)
    P = (2.0 / (1.0 + 0.05 * d2.min(axis=0))).astype(np.float32)
    Kf = rng.random(U.shape).astype(np.float32) * 3
    for arr in (U, P, Kf):
        arr[0, :, :] = arr[-1, :, :] = arr[:, 0, :] = arr[:, -1, :] = arr[:, :, 0] = arr[:, :, -1] = 0
    atoms5 = np.concatenate([pos, Z[:, None], rc[:, None]], axis=1).astype(np.float32).reshape(-1)
    return dict(U=U.reshape(-1), P=P.reshape(-1), K=Kf.reshape(-1), label=label.reshape(-1), atoms5=atoms5)


def kernels_fixture(path):
    import oracle
    oracle.build()
    R = oracle.RefKernels()
    NN, nA = 16, 5
    S = NN + 1
    S3 = S ** 3
    h = 0.25
    st = seeded_state(NN, nA, seed=7)
    out = {f"in_{k}": v for k, v in st.items()}
    out["NN"], out["h"], out["nAtoms"] = NN, h, nA
    blk, grid = 256, (S3 + 255) // 256
    half_dv, dtv = np.float32(0.06), np.float32(0.12 * h * h)
    Unew = np.zeros(S3, np.float32)
    R.launch("updateU", grid, blk, (st["U"], Unew, st["K"], st["P"], st["label"], S, half_dv, dtv), serial=True)
    out["out_updateU"], out["half_dv"], out["dtv"] = Unew, half_dv, dtv
    rho = np.zeros(S3, np.float32)
    R.launch("computeRho", grid, blk, (rho, st["U"], S3), serial=True)
    P2 = np.zeros(S3, np.float32)
    coeff = np.float32(2 * np.pi)
    R.launch("jacobiStep", grid, blk, (st["P"], P2, rho, S, np.float32(h * h), coeff), serial=True)
    out["out_jacobiStep"] = P2
    U0 = np.zeros(S3, np.float32); lab0 = np.zeros(S3, np.int32); K0 = np.zeros(S3, np.float32)
    best = np.zeros(S3, np.float32)
    R.launch("initTrial", grid, blk, (U0, lab0, K0, best, st["atoms5"], nA, S, np.float32(h), np.float32(h * h)),
             serial=True)
    out["out_initTrial_U"], out["out_initTrial_label"], out["out_initTrial_K"] = U0, lab0, K0
    K1 = np.zeros(S3, np.float32)
    R.launch("recomputeK", grid, blk, (K1, st["atoms5"], nA, S, np.float32(h), np.float32(h * h)), serial=True)
    out["out_recomputeK"] = K1
    lab = st["label"].copy()
    R.launch("boundaryEvolve", grid, blk,
             (st["U"], lab, st["atoms5"], nA, S, np.float32(h), np.float32(h * h), np.float32(h ** 3), np.float32(0.5)),
             serial=True)
    out["out_boundaryEvolve_inplace"] = lab
    F = np.zeros(nA * 3, np.float32)
    R.launch("computeForceAll", grid, blk,
             (st["U"], F, st["atoms5"], nA, S, np.float32(h), np.float32(h * h), np.float32(h ** 3)), serial=True)
    out["out_computeForceAll"] = F
    norms = np.zeros(nA, np.float32)
    np.add.at(norms, np.clip(st["label"], 0, nA - 1), st["U"] * st["U"] * np.float32(h ** 3))
    Un = st["U"].copy()
    Zeff = st["atoms5"].reshape(nA, 5)[:, 3].copy()
    R.launch("normalizeU", grid, blk, (Un, st["label"], norms, Zeff, S3, nA, np.float32(h ** 3)), serial=True)
    out["out_normalizeU"], out["norms_f32"] = Un, norms
    np.savez_compressed(path, **out)


def h2o_config(NN=32, scr=8.0):
    N2 = NN // 2
    return {"gridN": NN, "screen": scr, "atoms": [
        {"i": 13, "j": 14, "Z": 1, "el": "H", "rc": 0},
        {"i": N2, "j": N2, "Z": 2, "el": "O", "rc": 0.4},
        {"i": 19, "j": 14, "Z": 1, "el": "H", "rc": 0}]}


def run_fixture(reference, path):
    import cupy  # the stand-in
    cupy.SERIAL = True
    spec = importlib.util.spec_from_file_location("ref_solver", os.path.join(reference, "cloud", "solver.py"))
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)
    cfg = h2o_config()
    s = ref.RealQMSolver(cfg)
    res = s.run(total_steps=200, report_interval=100)
    keep = ("step", "E", "E_T", "E_eK", "E_ee", "E_KK", "E_bind")
    with open(path, "w") as f:
        json.dump({"config": cfg, "steps": 200, "label_semantics": "serial in-place (index order)",
                   "snapshots": [{k: r[k] for k in keep} for r in res],
                   "final_label_checksum": int(np.asarray(s.label, np.int64).sum()),
                   "final_U_sum": float(np.asarray(s.U, np.float64).sum())}, f, indent=1)


def hairpin_fixtures(reference, cfg_path, gold_path):
    sys.modules.setdefault("modal", types.SimpleNamespace(
        App=lambda *a, **k: types.SimpleNamespace(function=lambda *a, **k: (lambda f: f),
                                                  local_entrypoint=lambda *a, **k: (lambda f: f)),
        Image=types.SimpleNamespace(from_registry=lambda *a, **k: types.SimpleNamespace(
            pip_install=lambda *a, **k: types.SimpleNamespace(add_local_file=lambda *a, **k: None)))))
    spec = importlib.util.spec_from_file_location("ref_hairpin", os.path.join(reference, "cloud", "run_hairpin.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    cfg = mod.build_hairpin_config()
    with open(cfg_path, "w") as f:
        json.dump(cfg, f)
    with open(os.path.join(reference, "cloud", "hairpin_results.json")) as f:
        res = json.load(f)
    keep = ("step", "E", "E_T", "E_eK", "E_ee", "E_KK", "E_bind", "ms_per_step")
    with open(gold_path, "w") as f:
        json.dump({"source": "cloud/hairpin_results.json (reference A100 run)",
                   "snapshots": [{k: s[k] for k in keep} for s in res["snapshots"]],
                   "first_nucPos": res["snapshots"][0]["nucPos"],
                   "final_E": res["final_E"], "final_E_bind": res["final_E_bind"],
                   "final_nucPos": res["final_nucPos"]}, f)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("REALQM_REFERENCE_DIR", "/root/reference"))
    a = ap.parse_args()
    kernels_fixture(os.path.join(HERE, "solverpy_kernels_nn16.npz"))
    run_fixture(a.reference, os.path.join(HERE, "solverpy_run_h2o_nn32.json"))
    hairpin_fixtures(a.reference, os.path.join(HERE, "hairpin_config.json"), os.path.join(HERE, "hairpin_golden.json"))
    print("golden fixtures written to", HERE)
