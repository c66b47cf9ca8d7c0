"""The molecule.js page host (MoleculePage) on the GPU: its dynamics frames against the same host
logic driven by the oracle's restatement of the frames (an adapter with the Context methods the
host uses), and the headless slice buffer (rq_extract) against the fields it is cut from.

Frames are bit-exact between the two (test_gpu_mj.py) and the Hartree-gradient forces agree to
1e-9, so the nuclear positions after moves agree to 1e-7 cells and K (rebuilt from the
truncated positions) is bit-equal."""
import numpy as np
import pytest

import oracle as orc
from realmolecule_b200 import _lib as L

pytestmark = pytest.mark.gpu

NN, SCREEN = 40, 10.0
ROWS = [{"i": 20, "j": 20, "k": 20, "Z": 6, "Z_nuc": 6, "rc": 0.4},
        {"i": 23, "j": 17, "k": 20, "Z": 1, "Z_nuc": 1, "rc": 0.0},
        {"i": 17, "j": 17, "k": 20, "Z": 1, "Z_nuc": 1, "rc": 0.0}]


class OracleContext:
    """The Context methods MoleculePage uses, over oracle.MoleculeJsDriver."""

    def __init__(self, ref):
        self.ref = ref

    def step(self, n):
        for _ in range(n):
            self.ref.step()

    def energy(self):
        return np.zeros(L.ENERGY_LEN)

    def forces(self, method):
        r = self.ref
        F = np.zeros(r.nA * 3)
        orc.O().mj_force_gradP(r.P, orc.C.addressof(r.atoms), r.nA, r.S, np.float32(1 / r.hd), max(5, round(3.0 / r.hd)), F)
        return F.reshape(r.nA, 3)

    def set_atoms(self, rows):
        self.ref.set_positions(rows)

    def initialize(self):
        self.ref.initialize()


def pages(**kw):
    from realmolecule_b200.molecule_host import MoleculePage
    ref = orc.MoleculeJsDriver(NN, SCREEN, ROWS, steps_per_frame=kw.get("steps_per_frame"))
    ref.initialize()
    cpu = MoleculePage(ROWS, NN=NN, screen=SCREEN, context=OracleContext(ref), **kw)
    gpu = MoleculePage(ROWS, NN=NN, screen=SCREEN, **kw)
    gpu.ctx.initialize()
    gpu.ctx.upload(psi=ref.U, label=ref.label.astype(np.int32))
    return ref, cpu, gpu


def test_dynamics_frames_follow_the_restatement():
    ref, cpu, gpu = pages(steps_per_frame=5, dynamics=True, dt_nuc=40.0, no_auto_dynamics=True)
    for _ in range(6):  # forces and a move every second frame
        cpu.frame()
        gpu.frame()
    assert gpu.nuc_steps == cpu.nuc_steps == 3
    np.testing.assert_allclose(np.array(gpu.pos), np.array(cpu.pos), rtol=0, atol=1e-7)
    assert not np.allclose(np.array(gpu.pos), np.array([[r["i"], r["j"], r["k"]] for r in ROWS]))
    assert np.array_equal(gpu.ctx.download_K().view(np.uint32), ref.K.view(np.uint32))
    gpu.close()


def test_slice_buffer_and_restart():
    from realmolecule_b200.molecule_host import MoleculePage
    p = MoleculePage(ROWS, NN=NN, screen=SCREEN, steps_per_frame=5)
    p.initialize()
    for _ in range(2):
        p.frame()
    S, sk = NN + 1, NN // 2
    out = p.extract()
    assert out.shape == (3 * S * S + 2 * S,)
    st = p.ctx.download(psi=True, label=True)
    U = st["psi"].reshape(S, S, S)[:, :, sk]
    lab = st["label"].reshape(S, S, S)[:, :, sk]
    dens = out[:S * S].reshape(S, S)
    code = out[S * S:2 * S * S].reshape(S, S)
    inner = (slice(1, NN), slice(1, NN))
    assert np.array_equal(dens[inner], (U * U)[inner])
    Z = np.array([r["Z"] for r in ROWS], np.float32)
    assert np.array_equal(code[inner], (lab.astype(np.float32) + Z[lab] * np.float32(1000))[inner])
    bnd = out[2 * S * S:3 * S * S].reshape(S, S)
    diff_i = np.zeros((S, S), bool)  # a label change towards i+1 always marks a boundary
    diff_i[2:NN - 1, 1:NN] = lab[2:NN - 1, 1:NN] != lab[3:NN, 1:NN]
    assert set(np.unique(bnd)) <= {0.0, 1.0, 2.0} and diff_i.any() and (bnd[diff_i] > 0).all()
    K = p.ctx.download_K().reshape(S, S, S)
    assert np.array_equal(out[3 * S * S:3 * S * S + S], K[:, sk, sk])
    assert np.all(out[3 * S * S + S:] == 1.0)
    p.restartWithPositions([[21, 20, 20], [24, 17, 20], [17, 18, 20]])
    assert p.tStep == 0 and p.frame()["E"] is not None
    p.close()
