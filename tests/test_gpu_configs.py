"""Parity at the benchmark configurations themselves (new flavour, GPU through the C ABI against
the FP64 oracle of the same method, oracle.NewMethodDriver).

C1  -- H2O all-electron, 64^3 at h = 0.25 bohr, 10 jittered seeds, 4-level multigrid, the full
       3000 steps at dt = 0.2 h^2 in FP64: labels equal to the oracle's, energy components within
       1e-11 relative.
C3  -- three real instances of the 96-cluster batch (the smallest grid, a middle one and the
       largest cluster) stepped together in one batch: FP64 batch energies within 1e-11 relative
       of the oracle after 200 steps; the mixed-precision batch within 1e-6 relative.
Labels -- one level-set pass of the mixed path from an identical fp32 state (psi, labels, W)
       against the oracle's f32 form of the rule (orc_nm_evolve_f32): labels and W bit-exact; the
       same for the FP64 path against orc_nm_evolve.
"""
import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu


def _oracle_energies(ref):
    o = ref.energy()
    return np.array([o["E"], o["T"], o["EK"], o["EE"], o["KK"]])


def test_c1_h2o_fp64_3000_steps_against_the_oracle():
    from realmolecule_b200 import Context, configs as C, _lib as L
    g = C.h2o64()
    rows = C.to_domain_atoms(g)
    ref = orc.NewMethodDriver(g.NN, g.screen, rows)
    ref.initialize()
    ctx = Context(g.NN, g.screen, rows, flavor="new", precision="fp64")
    assert ctx.info().mg_levels == 4
    ctx.initialize()
    for _ in range(3000):
        ref.step()
    ctx.step(3000)
    st = ctx.download(psi=True, label=True)
    U, lab, _ = ref.state()
    assert np.array_equal(st["label"], lab)
    assert np.max(np.abs(st["psi"] - U)) <= 1e-10 * np.abs(U).max()
    e = ctx.energy()
    got = np.array([e[L.E_TOTAL], e[L.E_T], e[L.E_EK], e[L.E_EE], e[L.E_KK]])
    want = _oracle_energies(ref)
    assert np.all(np.abs(got - want) <= 1e-11 * np.abs(want)), (got, want)
    ctx.close()


def _three_clusters():
    from realmolecule_b200 import configs as C
    gs = C.clusters96()
    size = sorted((g.NN, len(g.elements), q) for q, g in enumerate(gs))
    picks = [size[0][2], size[len(size) // 4][2], size[-1][2]]  # smallest, a middle grid class, largest
    return [gs[q] for q in picks]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c3_three_cluster_instances_in_one_batch_against_the_oracle(precision):
    from realmolecule_b200 import configs as C, _lib as L
    from realmolecule_b200.batch import Batch
    gs = _three_clusters()
    inst = [{"NN": g.NN, "screen": g.screen, "atoms": C.to_domain_atoms(g)} for g in gs]
    assert len({g.NN for g in gs}) >= 2  # uneven grids in one batch
    b = Batch(inst, precision=precision)
    b.initialize()
    b.step(200)
    E = b.energy()
    b.close()
    tol = 1e-11 if precision == "fp64" else 1e-6
    for q, it in enumerate(inst):
        ref = orc.NewMethodDriver(it["NN"], it["screen"], it["atoms"])
        ref.initialize()
        for _ in range(200):
            ref.step()
        want = _oracle_energies(ref)
        got = E[q, [L.E_TOTAL, L.E_T, L.E_EK, L.E_EE, L.E_KK]]
        assert np.all(np.abs(got - want) <= tol * np.abs(want)), (q, got, want)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_one_label_pass_from_an_identical_state_is_bit_exact(precision):
    """The label pass of step s reads the psi the update of step s left (normalised) and the labels
    and W of step s-1; neither the pass nor anything after it in the step changes psi."""
    from realmolecule_b200 import Context, configs as C
    g = C.h2o64()
    rows = C.to_domain_atoms(g)
    ctx = Context(g.NN, g.screen, rows, flavor="new", precision=precision, label_interval=20)
    ctx.initialize()
    ctx.step(59)  # the next step (60) ends with a label pass
    before = ctx.download(psi=False, label=True, W=True)
    ctx.step(1)
    after = ctx.download(psi=True, label=True, W=True)
    lab = np.empty_like(before["label"])
    W = before["W"].copy()
    if precision == "mixed":
        orc.O().nm_evolve_f32(before["label"], lab, after["psi"], W, g.NN + 1, np.float32(0.5), np.float32(0.15))
    else:
        orc.O().nm_evolve(before["label"], lab, after["psi"], W, g.NN + 1, float(np.float32(0.5)),
                          float(np.float32(0.15)))
    assert np.array_equal(lab, after["label"])
    assert np.array_equal(W.view(np.uint32), after["W"].view(np.uint32))
    assert (lab != before["label"]).any()  # the pass moved some boundary
    ctx.close()
