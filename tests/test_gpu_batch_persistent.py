"""The persistent form of a batch period (one cooperative launch: blocks take chunks of
(instance, tile) items from one queue, an item waits only for its instance's previous phase)
against the per-kernel launches of the same schedule, and its bounded waits.

Bars: the same instances stepped 200 steps both ways -- FP64 energies within 1e-12 relative (the
two differ only in the order of the FP64 per-domain atomics), mixed within 1e-6; one kernel
launch per period instead of one per kernel.  Dependencies made to wait for a completion that
never comes give up after their limit: the launch ends, the next readout reports RQ_ETIMEOUT,
and the batch works again after re-initialisation."""
import numpy as np
import pytest

from test_gpu_batch import instances

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_persistent_matches_per_kernel(precision):
    from realmolecule_b200 import _lib as L
    from realmolecule_b200.batch import Batch
    E, launches = {}, {}
    for persistent in (0, 1):
        b = Batch(instances(), precision=precision, label_interval=10, label_until=60, batch_persistent=persistent)
        b.initialize()
        l0 = b.info()["kernel_launches"]
        b.step(200)
        E[persistent] = b.energy()
        launches[persistent] = b.info()["kernel_launches"] - l0
        b.close()
    tol = 1e-12 if precision == "fp64" else 1e-6
    for k in (L.E_T, L.E_EK, L.E_EE, L.E_TOTAL):
        np.testing.assert_allclose(E[1][:, k], E[0][:, k], rtol=tol, atol=tol)
    # one launch per 20-step period
    assert launches[1] < launches[0] / 10, launches


def test_persistent_wait_runs_out_and_recovers():
    from realmolecule_b200 import _lib as L
    from realmolecule_b200.batch import Batch
    b = Batch(instances(), precision="fp64", label_interval=20, batch_persistent=1)  # 20-step periods
    b.initialize()
    b.step(20)
    want = b.energy()
    b.set_wait(1_000_000, extra_arrivals=1)  # 1 ms; every dependency waits for a completion that never comes
    b.initialize()
    b.step(20)
    with pytest.raises(L.RqError) as err:
        b.energy()
    assert err.value.status == L.RQ_ETIMEOUT
    b.set_wait(2_000_000_000, 0)
    b.initialize()
    b.step(20)
    np.testing.assert_allclose(b.energy(), want, rtol=1e-12, atol=1e-12)
