"""Batched new-flavour instances (one launch per kernel over the (instance, tile) work list)
against the same instances stepped one by one through their own contexts.  Every instance runs
the same device bodies on the same data, so the FP64 batch agrees with the single contexts up to
the order of the FP64 per-domain atomics: labels equal, energies within 1e-11 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def instances(h=0.5):
    from realmolecule_b200 import configs as C
    out = []
    rng = np.random.default_rng(1)
    for q, NN in enumerate((32, 24, 40, 32)):
        g = C.h2o64(seed=q)
        g.NN, g.h = NN, h
        g.xyz = g.xyz @ C.random_rotation(rng).T
        g.seeds = g.seeds @ np.eye(3)
        out.append({"NN": NN, "screen": NN * h, "atoms": C.to_domain_atoms(g)})
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_single_contexts(precision):
    from realmolecule_b200 import Context, _lib as L
    from realmolecule_b200.batch import Batch
    inst = instances()
    b = Batch(inst, precision=precision, label_interval=10, label_until=60)
    b.initialize()
    b.step(120)
    Eb = b.energy()
    Fb = b.forces()
    for q, it in enumerate(inst):
        c = Context(it["NN"], it["screen"], it["atoms"], flavor="new", precision=precision, label_interval=10,
                    label_until=60)
        c.initialize()
        c.step(120)
        e = c.energy()
        tol = 1e-11 if precision == "fp64" else 1e-6
        for k in (L.E_T, L.E_EK, L.E_EE, L.E_KK, L.E_TOTAL):
            assert abs(Eb[q, k] - e[k]) <= tol * max(1.0, abs(e[k])), (q, k, Eb[q, k], e[k])
        F = c.forces(L.FORCE_ADJOINT) + c.nuclear_terms()[1]
        # fp32 fields: the two runs round psi differently wherever their FP64 domain sums (atomics in
        # a different order) differ in the last bit, ~1e-7 of the largest force
        np.testing.assert_allclose(Fb[q], F, rtol=1e-6, atol=1e-8 if precision == "fp64" else 1e-6)


def test_mixed_solve_matches_fp64_solve_to_1e6_ha():
    """The mixed solve (fp32 to its noise floor, then FP64 refinement of the same batch) reaches the
    FP64 solve's converged energies within 1e-6 Ha, instance by instance."""
    from realmolecule_b200.batch import Batch
    E = {}
    for p in ("mixed", "fp64"):
        b = Batch(instances(), precision=p, label_until=200)
        b.initialize()
        b.step(200)
        conv, E[p] = b.solve(1e-8, 40000, 100)
        assert (conv > 0).all(), (p, conv)
        info = b.info()
        assert info["instances"] == 4 and info["kernel_launches"] > 0
    assert np.max(np.abs(E["mixed"] - E["fp64"])) < 1e-6, (E["mixed"], E["fp64"])
