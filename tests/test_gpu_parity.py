"""Parity of the sm_100a path (through the C-ABI) with the CPU FP64 oracle.

Tolerance: relative Frobenius error <= 1e-10 on H, G (pre-swap), the swapped
system and the solution (the plain-path bar); the static diagonals to 1e-12.
"""
import os

import numpy as np
import pytest

import oracle
import refmetrics
from bem_mececcs_b200 import formats, meshgen
from bem_mececcs_b200.capi import BEM_ERR_DEGENERATE, BEM_ERR_SINGULAR, BemError, Context
from bem_mececcs_b200.solver import BemSolver, solve_dense
from gpu_util import rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _setup(s, d, ctx, gest_from_gpu=True):
    sol = BemSolver(s, ctx=ctx)
    hd, gd = sol.ghmatece(compute_gest=gest_from_gpu)
    sol.set_bc(d.kode, d.bc.astype(np.complex128), d.dam, d.rho)
    return sol, hd, gd


@pytest.mark.parametrize("n", [1, 2, 7, 63, 64, 65, 130, 257, 1000])
def test_lu_random(ctx, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    x = solve_dense(ctx, a, b)
    ref = np.linalg.solve(a, b)
    assert rel(x, ref) < 1e-11 * max(1.0, np.linalg.cond(a) / 100)


@pytest.mark.parametrize("scheme", ["cublas_pairs", "cublas", "f64_pairs", "one_panel"])
def test_lu_tall_panels_pairs(ctx, scheme):
    """n = 4000: the FP64 panels above 3440 rows are 32 columns wide, so two
    of them share one K = 64 trailing update (f64_pairs), the first panel's L
    read through the second's gather list.  Rows are shuffled so that every
    panel pivots across the pair; the result must not depend on the scheme:
    pairs on cuBLAS ZGEMM with the gathered L in a buffer (the default), one
    panel per cuBLAS update, pairs on the own DMMA kernel, or one panel at a
    time on it."""
    n = 4000
    rng = np.random.default_rng(40)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    a = a[rng.permutation(n)] * np.exp(rng.uniform(-3, 3, n))[:, None]  # uneven row scales: real pivoting
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    defaults = {k: ctx.get_option(k) for k in ("f64_cublas", "f64_pairs")}
    ctx.set_option("f64_cublas", scheme.startswith("cublas"))
    ctx.set_option("f64_pairs", scheme in ("cublas_pairs", "f64_pairs"))
    try:
        x = solve_dense(ctx, a, b)
    finally:
        for k, v in defaults.items():
            ctx.set_option(k, v)
    # normwise backward error at FP64 level, and the same solution as LAPACK's
    berr = np.linalg.norm(a @ x - b) / (np.linalg.norm(a) * np.linalg.norm(x) + np.linalg.norm(b))
    assert berr < 1e-15
    assert rel(x, np.linalg.solve(a, b)) < 1e-10


def test_lu_needs_pivoting(ctx):
    n = 200
    rng = np.random.default_rng(3)
    perm = rng.permutation(n)
    a = np.zeros((n, n), dtype=complex)
    a[np.arange(n), perm] = 1.0 + 2.0j   # zero diagonal almost everywhere
    a += 1e-3 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    b = rng.standard_normal(n) + 0j
    assert rel(solve_dense(ctx, a, b), np.linalg.solve(a, b)) < 1e-12


def test_lu_singular_reported(ctx):
    n = 96
    rng = np.random.default_rng(4)
    a = rng.standard_normal((n, n)) + 0j
    a[:, 40] = 0.0
    with pytest.raises(BemError) as e:
        solve_dense(ctx, a, np.ones(n, dtype=complex))
    assert e.value.code == BEM_ERR_SINGULAR


def test_static_diagonals_c1(ctx):
    s, d = meshgen.config_mesh("c1_240")
    p = oracle.OracleProblem(s, d)
    ohd, ogd, ohest = p.ghmatece(want_hest=True)
    sol, hd, gd = _setup(s, d, ctx)
    assert rel(hd, ohd) < 1e-12
    assert rel(gd, ogd) < 1e-12
    assert rel(sol.static_h(), ohest) < 1e-12


def test_dynamic_c1_parity(ctx):
    s, d = meshgen.config_mesh("c1_240")
    p = oracle.OracleProblem(s, d)
    p.ghmatece()
    fr = d.freqs[0]
    ozh, ozfi, ozh0, ozg0 = p.system(fr)
    sol, _, _ = _setup(s, d, ctx)
    sol.ghmatecd(fr, keep_preswap=True)
    zh0, zg0 = sol.get_preswap()
    assert rel(zh0, ozh0) < TOL
    assert rel(zg0, ozg0) < TOL
    zh, zfi = sol.get_system()
    assert rel(zh, ozh) < TOL and rel(zfi, ozfi) < TOL
    x = sol.linsolve()
    ox = oracle.zgesv(ozh, ozfi, use_openblas=False)
    assert rel(x, ox) < TOL
    disp, trac = sol.interec()
    assert rel(disp, ox) < TOL and np.array_equal(trac, d.bc.astype(complex))


def test_dynamic_mixed_kode(ctx):
    """KODE = 0 columns exercise the H/G column swap and the un-swap."""
    s, d = meshgen.config_mesh("c1_240")
    rng = np.random.default_rng(11)
    d.kode = (rng.random(3 * s.nbe) > 0.3).astype(np.int32)
    d.bc = rng.standard_normal(3 * s.nbe)
    p = oracle.OracleProblem(s, d)
    p.ghmatece()
    fr = 1.7
    ozh, ozfi, _, _ = p.system(fr)
    odisp, otrac, ox = p.solve(fr, use_openblas=False)
    sol, _, _ = _setup(s, d, ctx)
    sol.ghmatecd(fr)
    zh, zfi = sol.get_system()
    assert rel(zh, ozh) < TOL and rel(zfi, ozfi) < TOL
    x = sol.linsolve()
    assert rel(x, ox) < TOL
    disp, trac = sol.interec()
    assert rel(disp, odisp) < TOL and rel(trac, otrac) < TOL
    # the reference's own GPU-vs-CPU checks (-DTEST_CUDA) on the same arrays
    assert refmetrics.ghmatecd_zh_zfi(zh, ozh, zfi, ozfi, s.nbe)[2]
    assert refmetrics.zfi(x, ox)[2]


def test_golden_240_end_to_end(ctx, golden_dir):
    """The reference's own known-answer test (src/tests.sh:38-50) with the
    GPU boundary solution: N=240 > NBE=100 (enclosing elements), NPG=8."""
    s = formats.read_static(os.path.join(golden_dir, "ESOLO240E_-5+5.DAT"))
    d = formats.read_dynamic(os.path.join(golden_dir, "ESOLO240D_-5+5.DAT"), s.nbe)
    p = oracle.OracleProblem(s, d)
    ohd, ogd, _ = p.ghmatece()
    sol, hd, gd = _setup(s, d, ctx)
    assert rel(hd, ohd) < 1e-12 and rel(gd, ogd) < 1e-12
    assert refmetrics.ghmatece_h_g(hd, ohd, gd, ogd, s.nbe)[2]  # ASSERT_GHMATECE_H_G
    fr = d.freqs[0]
    disp, trac = sol.solve_frequency(fr)
    odisp, _, _ = p.solve(fr, use_openblas=False)
    assert rel(disp, odisp) < TOL
    assert refmetrics.zfi(disp, odisp)[2]  # ASSERT_ZFI
    zdsol, zssol = p.interior(fr, disp, trac)
    mine = formats.Results(fr, disp.reshape(-1, 3), trac.reshape(-1, 3),
                           zdsol.reshape(-1, 3), zssol.reshape(-1, 9))
    gold = formats.parse_results(os.path.join(golden_dir, "SSOLO240D_-5+5.SOL"))[0]
    err = formats.dtester_errors(mine, gold)
    assert all(v <= 1e-3 for v in err.values()), err


@pytest.mark.slow
def test_golden_2160_end_to_end(ctx, golden_dir):
    s = formats.read_static(os.path.join(golden_dir, "ESOLO2160E_-5+5.DAT"))
    d = formats.read_dynamic(os.path.join(golden_dir, "ESOLO2160D_-5+5.DAT"), s.nbe)
    sol, _, _ = _setup(s, d, ctx)
    fr = d.freqs[0]
    disp, trac = sol.solve_frequency(fr)
    p = oracle.OracleProblem(s, d)
    zdsol, zssol = p.interior(fr, disp, trac)
    mine = formats.Results(fr, disp.reshape(-1, 3), trac.reshape(-1, 3),
                           zdsol.reshape(-1, 3), zssol.reshape(-1, 9))
    gold = formats.parse_results(os.path.join(golden_dir, "SSOLO2160D_-5+5.SOL"))[0]
    err = formats.dtester_errors(mine, gold)
    assert all(v <= 1e-3 for v in err.values()), err


@pytest.mark.slow
def test_c2_2160_solution_parity(ctx):
    """48x45 jittered mesh, omega=2, n=6480: solution within 1e-10 of the oracle."""
    s, d = meshgen.config_mesh("c2_2160")
    p = oracle.OracleProblem(s, d)
    p.ghmatece()
    fr = d.freqs[0]
    ozh, ozfi, _, _ = p.system(fr)
    ox = oracle.zgesv(ozh, ozfi, use_openblas=True)
    sol, _, _ = _setup(s, d, ctx)
    sol.ghmatecd(fr)
    zh, zfi = sol.get_system()
    assert rel(zh, ozh) < TOL and rel(zfi, ozfi) < TOL
    x = sol.linsolve()
    assert rel(x, ox) < TOL


def test_degenerate_element_reported(ctx):
    s, d = meshgen.config_mesh("c1_240")
    # Collapse element 5 onto a line: its Jacobian vanishes (DET < 1e-5).
    c = s.cone[5] - 1
    s.cx[c[2]] = s.cx[c[1]]
    s.cy[c[2]] = s.cy[c[1]]
    s.cx[c[3]] = s.cx[c[0]]
    s.cy[c[3]] = s.cy[c[0]]
    with pytest.raises(BemError) as e:
        sol = BemSolver(s, ctx=ctx)
        sol.ghmatece()
    assert e.value.code == BEM_ERR_DEGENERATE
