"""The serving form (bem_server_*): continuous batching over resident meshes.

* a request's result is the same alone and in a mix of concurrent requests;
* a right-hand-side-only request (same mesh, material, omega and KODE, new
  traction patch) is solved with the cached factors and matches a fresh
  full solve;
* the plain form matches bem_ghmatecd + bem_linsolve;
* admission respects the HBM budget (evicting idle problems) and refuses a
  problem larger than the budget.
"""
import numpy as np
import pytest

import oracle
from bem_mececcs_b200 import capi, meshgen, serve
from bem_mececcs_b200.solver import BemSolver
from gpu_util import rel

pytestmark = pytest.mark.gpu

MAT = (1.0, 0.25, 0.01, 1.0)
TOL = 1e-10


def _mesh(nx, ny, seed):
    return meshgen.enclosed_grid(nx, ny, jitter=0.10, seed=seed, depth=2.5, layers=4)


def _bc(m, cx, cy, rad):
    r = serve.Request(0.0, (0, 0), 0, 0.0, MAT, (cx, cy, rad))
    return serve.request_bc(m, r)


def test_alone_equals_in_mix_and_rhs_reuse():
    mA, mB, mC = _mesh(12, 10, 1), _mesh(16, 15, 2), _mesh(20, 18, 3)
    bcR, kode = _bc(mB, 0.5, -0.5, 1.2)
    frR = 1.3
    # alone
    srv = serve.Server(form="mixed", refine=3)
    b = srv.add_mesh(mB)
    dR, tR, info = srv.wait(srv.submit(b, MAT, frR, bcR, kode))
    assert not info["rhs_only"]
    srv.close()
    # in a mix: other meshes and omegas around it, all submitted at once
    srv = serve.Server(form="mixed", refine=3)
    a, b, c = srv.add_mesh(mA), srv.add_mesh(mB), srv.add_mesh(mC)
    ids = []
    for k, (mid, m) in enumerate([(a, mA), (c, mC), (a, mA), (c, mC)]):
        bc, kd = _bc(m, 0.3 * k, -0.2 * k, 1.0 + 0.2 * k)
        ids.append(srv.submit(mid, MAT, 0.7 + 1.1 * k, bc, kd))
    rid = srv.submit(b, MAT, frR, bcR, kode)
    ids.append(srv.submit(c, MAT, 4.0, *_bc(mC, 1.0, 1.0, 1.5)))
    dM, tM, _ = srv.wait(rid)
    for i in ids:
        srv.wait(i)
    st = srv.stats()
    assert st["max_busy"] >= 2 and st["completed"] == 6
    assert rel(dM, dR) < TOL and rel(tM, tR) < TOL
    # right-hand-side only: same problem, new patch -> cached factors
    bc2, _ = _bc(mB, -1.0, 1.0, 1.7)
    d2, t2, info2 = srv.wait(srv.submit(b, MAT, frR, bc2, kode))
    assert info2["rhs_only"]
    srv.close()
    # against a fresh full solve and the FP64 oracle
    sol = BemSolver(mB)
    sol.ghmatece()
    sol.set_bc(kode, bc2, MAT[2], MAT[3])
    d2f, _ = sol.solve_frequency(frR)
    sol.ctx.close()
    assert rel(d2, d2f) < TOL
    dyn = meshgen.traction_patch(mB, freqs=(frR,))
    dyn.kode[:] = kode
    dyn.bc = bcR
    od, ot, _ = oracle.OracleProblem(mB, dyn).solve(frR, use_openblas=False)
    assert rel(dR, od) < TOL and rel(tR, ot) < TOL


def test_plain_form_matches_linsolve():
    m = _mesh(16, 15, 5)
    bc, kode = _bc(m, 0.0, 0.0, 1.0)
    srv = serve.Server(form="plain")
    mid = srv.add_mesh(m)
    d, t, _ = srv.wait(srv.submit(mid, MAT, 2.2, bc, kode))
    bc2, _ = _bc(m, 1.0, -1.0, 1.3)
    d2, t2, info2 = srv.wait(srv.submit(mid, MAT, 2.2, bc2, kode))
    assert info2["rhs_only"]
    srv.close()
    sol = BemSolver(m)
    sol.ghmatece()
    sol.set_bc(kode, bc, MAT[2], MAT[3])
    df, tf = sol.solve_frequency(2.2)
    sol.set_bc(kode, bc2, MAT[2], MAT[3])
    d2f, t2f = sol.solve_frequency(2.2)
    sol.ctx.close()
    assert rel(d, df) < TOL and rel(t, tf) < TOL
    assert rel(d2, d2f) < TOL and rel(t2, t2f) < TOL


def test_admission_by_footprint():
    ms = [_mesh(16, 15, s) for s in (11, 12, 13)]
    srv0 = serve.Server(form="mixed")
    mid = srv0.add_mesh(ms[0])
    bc, kode = _bc(ms[0], 0, 0, 1)
    _, _, info = srv0.wait(srv0.submit(mid, MAT, 1.0, bc, kode))
    one = info["bytes"]
    srv0.close()
    # room for one problem at a time: the three run one after another
    srv = serve.Server(form="mixed", budget_bytes=1.5 * one)
    ids = []
    for m in ms:
        k = srv.add_mesh(m)
        bc, kode = _bc(m, 0, 0, 1)
        ids.append(srv.submit(k, MAT, 1.5, bc, kode))
    for i in ids:
        srv.wait(i)
    st = srv.stats()
    assert st["completed"] == 3 and st["evictions"] >= 2
    assert st["peak_bytes"] <= 1.5 * one and st["max_busy"] == 1
    # a problem bigger than the whole budget is refused
    big = srv.add_mesh(_mesh(40, 36, 14))
    bcb, kb = _bc(_mesh(40, 36, 14), 0, 0, 1)
    with pytest.raises(capi.BemError) as e:
        srv.wait(srv.submit(big, MAT, 1.0, bcb, kb))
    assert e.value.code == capi.BEM_ERR_NOMEM
    srv.close()


@pytest.mark.parametrize("form", ["mixed", "plain"])
def test_same_mesh_sweep_batched_in_lockstep(form):
    """Requests for one mesh, material and load at several omegas, submitted
    at once, run as lockstep batches in one slot (the sweep's form); each
    result equals the same request solved alone, and the batch's problems
    are not kept as cached factors."""
    m = _mesh(14, 12, 4)
    bc, kode = _bc(m, 0.0, 0.0, 1.5)
    freqs = [0.4, 0.9, 1.7, 2.6, 3.3, 4.8, 6.1, 7.7, 9.5]
    srv = serve.Server(form=form, refine=3)
    mid = srv.add_mesh(m)
    alone = [srv.wait(srv.submit(mid, MAT, f, bc, kode))[:2] for f in freqs]
    srv.close()
    srv = serve.Server(form=form, refine=3)
    mid = srv.add_mesh(m)
    ids = [srv.submit(mid, MAT, f, bc, kode) for f in freqs]
    got = [srv.wait(i)[:2] for i in ids]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(freqs) and st["max_busy"] >= 2  # several problems in flight together
    for (d0, t0), (d1, t1) in zip(alone, got):
        assert rel(d1, d0) < TOL and rel(t1, t0) < TOL
