"""The restated TEST_CUDA checks (tests/refmetrics.py) on the oracle: the
oracle against itself passes each, and a difference planted just above each
tolerance, in the shape the reference's metric measures, fails it."""
import numpy as np

import oracle
import refmetrics
from bem_mececcs_b200 import meshgen


def _problem():
    s, d = meshgen.config_mesh("c1_240")
    p = oracle.OracleProblem(s, d)
    hd, gd, _ = p.ghmatece()
    zh, zfi, _, _ = p.system(1.0)
    disp, trac, x = p.solve(1.0, use_openblas=False)
    return s, hd, gd, zh, zfi, x


def test_identical_results_pass_every_check():
    s, hd, gd, zh, zfi, x = _problem()
    assert refmetrics.ghmatece_h_g(hd, hd, gd, gd, s.nbe)[2]
    assert refmetrics.ghmatecd_zh_zfi(zh, zh, zfi, zfi, s.nbe)[2]
    assert refmetrics.zfi(x, x)[2]
    assert refmetrics.zdsol(x[:30], x[:30])[2]


def test_planted_differences_fail_their_check():
    s, hd, gd, zh, zfi, x = _problem()
    nbe, nn = s.nbe, 3 * s.nbe
    # HESTdiag: spread 1.2e-5 over one element's 9 entries (each only 1.3e-6)
    h2 = hd.copy()
    h2[9 * 7: 9 * 8] += 1.2e-5 / 9
    v, eps, ok = refmetrics.ghmatece_h_g(h2, hd, gd, gd, nbe)
    assert not ok and v > eps
    # ZH: a column whose 1-norm of the difference passes 1.5e-6 NBE, entries far below it
    z2 = zh.reshape(nn, nn, order="F").copy()
    z2[:, 11] += 1.6e-6 * nbe / nn
    v, eps, ok = refmetrics.ghmatecd_zh_zfi(z2, zh, zfi, zfi, nbe)
    assert not ok and eps == 1.5e-6 * nbe and np.abs(z2 - zh.reshape(nn, nn, order="F")).max() < eps / 100
    # ZFI alone
    f2 = zfi.copy()
    f2[3] += 2.0 * 1.5e-6 * nbe
    assert not refmetrics.ghmatecd_zh_zfi(zh, zh, f2, zfi, nbe)[2]
    # the solution and the interior displacements: one entry just past each bound
    x2 = x.copy()
    x2[5] += 1.3e-6
    assert not refmetrics.zfi(x2, x)[2] and not refmetrics.zdsol(x2[:30], x[:30])[2]
    x3 = x.copy()
    x3[5] += 1.1e-6
    assert refmetrics.zfi(x3, x)[2] and not refmetrics.zdsol(x3[:30], x[:30])[2]
