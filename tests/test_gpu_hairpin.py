"""The reference's only recorded solver output, reproduced through the drop-in RealQMSolver.

cloud/hairpin_results.json holds 10 snapshots (every 1000 steps) of the 267-atom solvated hairpin
job (cloud/run_hairpin.py:21-182; NN = 300, dynamics on, forces every 500 steps) run by the
reference on an A100.  That run sums norms and energies with f32 atomics in arbitrary order and
relabels in place while neighbours read labels, so it is not reproducible bit for bit even on
its own hardware.  This implementation relabels from a snapshot (deterministic), so the two
label fields part early; the largest gaps seen on B200 are E_T 3.7e-4 relative (step 2000),
E_ee 1.1e-4, E 1.0e-4, E_eK 5.1e-5, E_KK 1.5e-5, nuclear positions 0.02 cells.  Bar used
here: E_T within 5e-4 relative at every snapshot, E, E_eK and E_ee within 2e-4, E_KK within
5e-5, final nuclear positions within 0.05 grid cells (the reference's atoms moved up to 0.41
cells over the run).
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_hairpin_trajectory_matches_reference_a100_run():
    from realmolecule_b200 import RealQMSolver
    with open(os.path.join(GOLD, "hairpin_config.json")) as f:
        cfg = json.load(f)
    with open(os.path.join(GOLD, "hairpin_golden.json")) as f:
        gold = json.load(f)
    s = RealQMSolver(cfg)
    s.set_fold_atoms(cfg["fold_atoms"])
    res = s.run(total_steps=10000, report_interval=1000)
    assert [r["step"] for r in res] == [g["step"] for g in gold["snapshots"]]
    for r, g in zip(res, gold["snapshots"]):
        for k, bar in (("E_T", 5e-4), ("E_eK", 2e-4), ("E_ee", 2e-4), ("E", 2e-4)):
            assert abs(r[k] - g[k]) <= bar * abs(g[k]), (r["step"], k, r[k], g[k])
        assert abs(r["E_KK"] - g["E_KK"]) <= 5e-5 * abs(g["E_KK"]), (r["step"], r["E_KK"], g["E_KK"])
    assert np.abs(s.atom_pos - np.array(gold["final_nucPos"])).max() < 0.05
