"""molecule.js flavour against a number the reference itself holds.

molecule.js corrects the energy of every bare hydrogen by a table of "raw" single-atom values,
H_RAW = {100: [0.5, -1.0], 200: [0.503, -1.028], 300: [0.5, -1.0]} (molecule.js:3133): the E_T
and E_eK that the page's own method gives for one isolated H, against the exact 0.5 / -1.0.  The
NN = 100 and 300 entries are the exact values themselves (they correct nothing).  The NN = 200
entry is a measurement, and it is the single-atom test page test_1atom.html (NN = 200, screen
10 bohr, one H at the centre with r_c = 0.1, 10000 steps per run; test_1atom.html:19-27) run to
convergence: its raw E_T and E_eK (the per-domain sums before the correction), truncated to the
table's three decimals, are the table's 0.503 and -1.028.  This runs that page through the page
host (MoleculePage.from_page) on the GPU for 40000 steps.  The page switches nuclear dynamics on
after its 10000 steps; a single atom at a grid point feels no net force, so the run keeps the
dynamics off (NO_AUTO_DYNAMICS) and only the ITP frames continue.
"""
import math

import pytest

pytestmark = pytest.mark.gpu


def _trunc3(x):
    return math.trunc(x * 1000.0) / 1000.0


def test_single_h_page_reproduces_h_raw_200():
    from realmolecule_b200.molecule_host import MoleculePage
    page = {"USER_NN": 200, "USER_ATOMS": [{"i": 100, "j": 100, "Z": 1, "el": "H"}], "USER_SCREEN": 10,
            "USER_STEPS": 40000, "USER_Z": [1], "USER_RC": [0.1], "NO_AUTO_DYNAMICS": True}
    pg = MoleculePage.from_page(page)
    pg.initialize()
    while pg.phase == 0:
        pg.frame()
    _, pd = pg.ctx.energy(per_domain=True)
    T_raw, EK_raw = float(pd[0, 1]), float(pd[0, 2])
    pg.close()
    assert pg.phase_steps == 40000
    assert _trunc3(T_raw) == 0.503 and _trunc3(EK_raw) == -1.028, (T_raw, EK_raw)
