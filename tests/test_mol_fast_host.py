"""CPU checks of the mol_fast.js restatement (oracle.MolFastDriver) and of the page helpers:
the f32 workgroup-tree reduction against an FP64 sum of the same per-cell terms, the
normalisation hitting each occupation target, the per-electron V-cycle touching only that
electron's interior potential, and the page configurations' JavaScript rounding."""
import math

import numpy as np

import oracle as orc
from realmolecule_b200 import configs

NUC = [{"i": 10, "j": 12, "k": 12, "Z": 2, "rc": 0.4}, {"i": 15, "j": 12, "k": 12, "Z": 1}]


def driver(**kw):
    d = orc.MolFastDriver(NUC, NN=24, screen=8.0, norm_targets=[2, 1], **kw)
    d.initialize()
    return d


def interior(a, S):
    return a.reshape(S, S, S)[1:-1, 1:-1, 1:-1]


def test_tree_reduction_matches_fp64_sum():
    d = driver()
    d.do_steps(7)
    c, S, h3 = d.cur, d.S, np.float32(d.p.h3)
    orc.O().mf_reduce(d.pp, d.U[c], d.W[c], d.P[c], d.K, d.sums)
    for m in range(d.n):
        u = interior(d.U[c][m * d.S3:(m + 1) * d.S3], S)
        exact = float(np.sum((u.astype(np.float32) * u * h3).astype(np.float64)))
        assert abs(float(d.sums[m]) - exact) <= 2e-6 * exact


def test_normalisation_hits_the_targets():
    d = driver()
    d.do_steps(40)  # the last step reduces and normalises
    for m, tg in enumerate((2, 1)):
        u = interior(d.U[d.cur][m * d.S3:(m + 1) * d.S3], d.S).astype(np.float64)
        assert abs(np.sum(u * u) * d.h3v - tg) < 1e-5 * tg


def test_vcycle_touches_only_its_electrons_interior():
    d = driver()
    d.do_steps(10)
    c, S = d.cur, d.S
    U, P = d.U[c].copy(), d.P[c].copy()
    orc.O().mf_vcycle(d.pp, U, P, 0, 10)
    diff = (P != d.P[c]).reshape(d.n, S, S, S)
    assert diff[0, 1:-1, 1:-1, 1:-1].any()
    assert not diff[1].any()
    assert not diff[0, 0].any() and not diff[0, -1].any() and not diff[0, :, 0].any() and not diff[0, :, :, -1].any()
    assert np.array_equal(U, d.U[c])


def test_page_configs_round_like_javascript():
    assert configs._js_round(2.5) == 3 and configs._js_round(-2.5) == -2
    h2 = configs.mol_fast_h2_page()
    assert [a["i"] for a in h2["nuclei"]] == [86, 114]
    ch4 = configs.mol_fast_ch4_page()
    assert ch4["nuclei"][1] == {"i": 134, "j": 100, "k": 100, "Z": 1, "rc": 0.0}
    assert ch4["norm_targets"] == [4, 1, 1, 1, 1]
