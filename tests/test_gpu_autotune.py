"""The batch autotuner (rq_batch_autotune) and the runtime march tile it picks.

Bars: every march tile gives the same FP64 batch to 1e-12 relative (the tile only changes which
thread computes which point and the order of the FP64 per-domain atomics); the autotuner reports
all 12 tile x launch candidates (6 where the device has no cooperative launch) and 7 smoother
candidates with positive times and convergence factors in (0, 1); a tuned batch and an untuned
one converge to the same energies within 1e-7 Ha; the reported choice works as configuration."""
import numpy as np
import pytest

from test_gpu_batch import instances

pytestmark = pytest.mark.gpu


def test_march_tiles_give_the_same_batch():
    from realmolecule_b200.batch import Batch
    E = []
    for tile in (4 | (16 << 8), 5 | (8 << 8), 4 | (32 << 8), 5 | (1 << 8)):
        b = Batch(instances(), precision="fp64", label_interval=10, label_until=60, batch_tile=tile)
        b.initialize()
        b.step(120)
        E.append(b.energy())
        b.close()
    for e in E[1:]:
        np.testing.assert_allclose(e, E[0], rtol=1e-12, atol=1e-12)


def test_autotune_reports_and_keeps_the_fixed_point():
    from realmolecule_b200.batch import Batch
    b = Batch(instances(), precision="fp64", label_until=1)
    b.initialize()
    rep = b.autotune()
    assert len(rep["tiles"]) in (6, 12) and len(rep["smoothers"]) == 7, rep
    assert all(t["ms_per_step"] > 0 for t in rep["tiles"])
    assert all(0 < s["rho"] < 1 and s["ms_per_cycle"] > 0 for s in rep["smoothers"])
    assert set(rep["config"]) == {"batch_tile", "batch_persistent", "mg_pre", "mg_post", "mg_coarse_sweeps"}
    conv, E = b.solve(1e-9, 40000, 100)
    assert (conv > 0).all()
    ref = Batch(instances(), precision="fp64", label_until=1)
    ref.initialize()
    conv0, E0 = ref.solve(1e-9, 40000, 100)
    assert (conv0 > 0).all()
    assert np.abs(E - E0).max() < 1e-7, (E, E0)
    again = Batch(instances(), precision="fp64", label_until=1, **rep["config"])
    again.initialize()
    again.step(40)
    assert np.isfinite(again.energy()).all()
