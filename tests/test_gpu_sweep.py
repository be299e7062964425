"""The batching and precision forms (bem_sweep) against the FP64 oracle.

Plain form: FP64 batched assembly + lockstep FP64 LU, <= 1e-10 relative.
Mixed form: FP32 LU on TF32 tensor cores + FP64 iterative refinement; the
target is <= 1e-8 relative error on the solution; with 3 refinement steps it
reaches the FP64 level, checked here at 1e-10.
"""
import numpy as np
import pytest

import oracle
from bem_mececcs_b200 import meshgen
from bem_mececcs_b200.capi import Context
from bem_mececcs_b200.solver import BemSolver
from gpu_util import rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    s, d = meshgen.config_mesh("c1_240")
    p = oracle.OracleProblem(s, d)
    p.ghmatece()
    ctx = Context(0)
    sol = BemSolver(s, ctx=ctx)
    sol.ghmatece(compute_gest=True)
    sol.set_bc(d.kode, d.bc.astype(np.complex128), d.dam, d.rho)
    yield s, d, p, sol
    ctx.close()


FREQS = [0.1, 0.37, 1.0, 2.5, 6.0, 10.0, 0.8]


def _oracle_x(p, fr):
    zh, zfi, _, _ = p.system(fr)
    return oracle.zgesv(zh, zfi, use_openblas=False)


@pytest.mark.parametrize("batch", [1, 3, 8])
def test_sweep_plain_batched(c1, batch):
    s, d, p, sol = c1
    x, _ = sol.sweep(FREQS, form="plain", batch=batch)
    for i, fr in enumerate(FREQS):
        assert rel(x[i], _oracle_x(p, fr)) < 1e-10, (batch, fr)


@pytest.mark.parametrize("batch", [1, 4, 8])
def test_sweep_mixed_refined(c1, batch):
    s, d, p, sol = c1
    x, corr = sol.sweep(FREQS, form="mixed", batch=batch, refine=3)
    for i, fr in enumerate(FREQS):
        e = rel(x[i], _oracle_x(p, fr))
        assert e < 1e-10, (batch, fr, e)
        assert corr[i] < 1e-9


def test_sweep_mixed_refinement_converges(c1):
    """No refinement: the FP32/TF32 LU alone is far from 1e-8; each FP64
    refinement step shrinks the error."""
    s, d, p, sol = c1
    errs = []
    for it in range(0, 4):
        x, _ = sol.sweep(FREQS[:2], form="mixed", batch=2, refine=it)
        errs.append(max(rel(x[i], _oracle_x(p, fr)) for i, fr in enumerate(FREQS[:2])))
    assert errs[0] > 1e-7
    assert errs[1] < errs[0] * 1e-2 and errs[2] < errs[1] and errs[3] < 1e-10, errs


def test_sweep_matches_single_solve(c1):
    s, d, p, sol = c1
    x, _ = sol.sweep([1.3], form="plain", batch=1)
    sol.ghmatecd(1.3)
    xs = sol.linsolve()
    assert rel(x[0], xs) < 1e-13


@pytest.mark.slow
def test_sweep_mixed_c2_2160():
    s, d = meshgen.config_mesh("c2_2160")
    ctx = Context(0)
    sol = BemSolver(s, ctx=ctx)
    sol.ghmatece(compute_gest=True)
    sol.set_bc(d.kode, d.bc.astype(np.complex128), d.dam, d.rho)
    freqs = [0.5, 2.0, 8.0]
    xm, corr = sol.sweep(freqs, form="mixed", batch=3, refine=3)
    xp, _ = sol.sweep(freqs, form="plain", batch=3)
    p = oracle.OracleProblem(s, d)
    p.ghmatece()
    ox = oracle.zgesv(*p.system(2.0)[:2], use_openblas=True)
    assert rel(xp[1], ox) < 1e-10
    for i in range(3):
        assert rel(xm[i], xp[i]) < 1e-8, (freqs[i], rel(xm[i], xp[i]))
    ctx.close()


@pytest.mark.parametrize("batch", [1, 4])
def test_sweep_mixed_cta_pair_update(c1, batch):
    """The FP32 trailing update by CTA pairs (option tc_pair: tcgen05
    cta_group::2, each pair one 128 x 128 complex tile) gives the refined
    solution at the FP64 level, as the one-CTA update does, and its
    unrefined FP32 solution is as close to the oracle's."""
    s, d, p, sol = c1
    default = sol.ctx.get_option("tc_pair")
    try:
        sol.ctx.set_option("tc_pair", False)
        x1, _ = sol.sweep(FREQS, form="mixed", batch=batch, refine=0)
        sol.ctx.set_option("tc_pair", True)
        x2, _ = sol.sweep(FREQS, form="mixed", batch=batch, refine=0)
        x3, corr = sol.sweep(FREQS, form="mixed", batch=batch, refine=3)
    finally:
        sol.ctx.set_option("tc_pair", default)
    for i, fr in enumerate(FREQS):
        ox = _oracle_x(p, fr)
        e1, e2 = rel(x1[i], ox), rel(x2[i], ox)
        assert e2 < 10 * max(e1, 1e-7), (batch, fr, e1, e2)
        assert rel(x3[i], ox) < 1e-10, (batch, fr)
        assert corr[i] < 1e-9


def test_small_clusters_same_factors(c1):
    """n = 720: the panel cluster shrinks from 16 CTAs to 4 (180 rows per
    CTA).  The pivots and arithmetic of a column step do not depend on how
    the rows are split, so both give the oracle's solution at 1e-10 and agree
    with each other to rounding."""
    s, d, p, sol = c1
    xs = {}
    for on in (True, False):
        sol.ctx.set_option("small_clusters", on)
        xs[on], _ = sol.sweep(FREQS[:3], form="plain", batch=3)
    sol.ctx.set_option("small_clusters", True)
    for i, fr in enumerate(FREQS[:3]):
        assert rel(xs[True][i], _oracle_x(p, fr)) < 1e-10
        assert rel(xs[True][i], xs[False][i]) < 1e-13


@pytest.mark.parametrize("tslu", [True, False], ids=["tournament", "grid_panel"])
def test_tall_fp32_panels(tslu):
    """n = 7500: the first FP32 panels are taller than one 16-CTA cluster
    holds (about 6900 rows), so they are factored by tournament pivoting
    (panel_tslu) or by the grid-barrier kernel.  Either way the refined mixed
    solution reaches the FP64 level of the plain path, which keeps partial
    pivoting."""
    from bem_mececcs_b200 import serve
    nx, ny = serve.grid_for(2500)
    m = meshgen.enclosed_grid(nx, ny, jitter=0.10, seed=9, depth=2.5, layers=4)
    d = meshgen.traction_patch(m, radius=2.0)
    sol = BemSolver(m)
    sol.ghmatece()
    sol.set_bc(d.kode, d.bc, d.dam, d.rho)
    assert sol.nn > 7000
    freqs = [0.7, 3.1]
    xp, _ = sol.sweep(freqs, form="plain", batch=2)
    sol.ctx.set_option("panel_tslu", tslu)
    xm, corr = sol.sweep(freqs, form="mixed", batch=2, refine=3)
    for i in range(len(freqs)):
        assert rel(xm[i], xp[i]) < 1e-10, (tslu, freqs[i])
        assert corr[i] < 1e-9
    sol.close()


def test_two_contexts_two_threads_other_sizes():
    """Two contexts driven from two host threads at once, on meshes of other
    sizes, so that the same kernels launch concurrently with other dynamic
    shared-memory sizes (the limit is a process-wide kernel attribute; it is
    only ever raised).  Every sweep must succeed and equal the same sweep run
    alone."""
    import threading
    meshes = [meshgen.enclosed_grid(nx, ny, jitter=0.10, seed=sd, depth=2.5, layers=4)
              for nx, ny, sd in ((16, 15, 21), (30, 27, 22))]
    sols, alone = [], []
    freqs = [0.6, 1.9, 3.3]
    for m in meshes:
        d = meshgen.traction_patch(m, radius=2.0)
        sol = BemSolver(m)
        sol.ghmatece()
        sol.set_bc(d.kode, d.bc, d.dam, d.rho)
        sols.append(sol)
        for form in ("mixed", "plain"):
            alone.append(sol.sweep(freqs, form=form, batch=3, refine=2)[0])
    errors, got = [], {}

    def run(i):
        try:
            for rnd in range(4):
                for j, form in enumerate(("mixed", "plain")):
                    got[(i, j, rnd)] = sols[i].sweep(freqs, form=form, batch=3, refine=2)[0]
        except Exception as e:  # reported below
            errors.append(e)

    th = [threading.Thread(target=run, args=(i,)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for s in sols:
        s.close()
    assert not errors, errors[0]
    for (i, j, rnd), x in got.items():
        assert rel(x, alone[2 * i + j]) < 1e-12, (i, j, rnd)


@pytest.mark.parametrize("form", ["mixed", "plain"])
def test_sweep_async_matches_sweep(c1, form):
    """bem_sweep_async: three sweeps in flight on one context, each into its
    own page-locked buffer, then one bem_sync; every buffer equals what
    bem_sweep returns for the same frequencies."""
    import torch
    from bem_mececcs_b200 import capi
    s, d, p, sol = c1
    groups = [FREQS[0:3], FREQS[3:6], FREQS[4:7]]
    want = [sol.sweep(g, form=form, batch=3, refine=2)[0] for g in groups]
    zge, zcs, zcp = sol.material
    zg, zc, zp = (capi.f64([z.real, z.imag]) for z in (zge, zcs, zcp))
    cc = capi.f64(sol.c)
    fm = capi.BEM_FORM_MIXED if form == "mixed" else capi.BEM_FORM_PLAIN
    bufs = [torch.empty(3 * sol.nn * 16, dtype=torch.uint8, pin_memory=True).numpy().view(np.complex128)
            for _ in groups]
    frs = [capi.f64(g) for g in groups]
    for fr, b in zip(frs, bufs):
        sol.ctx.check(sol.ctx.L.bem_sweep_async(sol.ctx.h, capi.ptr(zg), capi.ptr(zc), capi.ptr(zp), capi.ptr(cc),
                                                capi.ptr(fr), 3, fm, 3, 2, capi.ptr(b)), "bem_sweep_async")
    sol.ctx.sync()
    for w, b in zip(want, bufs):
        assert rel(b.reshape(3, sol.nn), w) < 1e-12
