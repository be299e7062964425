"""Failure paths on the GPU, made to happen without faulting or hanging it.

* Bounded device waits: with the context's wait limit at 30 ms, a bulk-copy
  mbarrier that no copy completes and a grid barrier that one CTA too few
  reach both give up, the call reports BEM_ERR_TIMEOUT well inside the 2 s
  default, and the same context then solves a problem correctly (the status
  is cleared by the next call).  The limit also holds for the product
  kernels: a full solve under the 30 ms limit is unaffected.
* The two seam entries that the reference's Fortran calls concurrently from
  two OpenMP sections (src/Ghmatece.for:202-242: cuda_ghmatece_ in one,
  GEST_SINGULAR + cuda_send_gest_data_ in the other) are called from two
  host threads at once, several times; the solution that depends on both
  diagonals must match the oracle at 1e-10 every time.
"""
import ctypes
import threading
import time

import numpy as np
import pytest

import oracle
from bem_mececcs_b200 import capi, host, meshgen
from bem_mececcs_b200.capi import BEM_ERR_ARG, BEM_ERR_TIMEOUT, BemError, Context
from bem_mececcs_b200.solver import BemSolver
from gpu_util import rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


def test_wait_limit_option_range():
    ctx = Context(0)
    assert ctx.get_option("wait_limit_ms") == 2000
    for bad in (0, -5, 60001):
        with pytest.raises(BemError) as e:
            ctx.set_option("wait_limit_ms", bad)
        assert e.value.code == BEM_ERR_ARG
    ctx.set_option("wait_limit_ms", 30)
    assert ctx.get_option("wait_limit_ms") == 30
    ctx.close()


@pytest.mark.parametrize("which", [0, 1], ids=["mbarrier", "grid_barrier"])
def test_bounded_wait_gives_up_and_context_survives(which):
    s, d = meshgen.config_mesh("c1_240")
    sol = BemSolver(s)
    sol.ghmatece()
    sol.set_bc(d.kode, d.bc, d.dam, d.rho)
    want = sol.solve_frequency(1.0)

    sol.ctx.set_option("wait_limit_ms", 30)
    t0 = time.perf_counter()
    rc = sol.ctx.wait_selftest(which)
    dt = time.perf_counter() - t0
    assert rc == BEM_ERR_TIMEOUT, capi.lib().bem_status_string(rc)
    assert 0.02 < dt < 1.0  # the 30 ms limit, not the 2 s default
    assert b"timed out" in sol.ctx.L.bem_last_error(sol.ctx.h)

    # the context is usable: a full solve under the same short limit
    got = sol.solve_frequency(1.0)
    assert rel(got[0], want[0]) < 1e-14 and rel(got[1], want[1]) < 1e-14
    x, _ = sol.sweep([0.5, 1.0], form="mixed", batch=2, refine=3)
    assert np.all(np.isfinite(x))
    assert sol.ctx.L.bem_wait_selftest(sol.ctx.h, 2) == BEM_ERR_ARG
    sol.close()


def test_seam_static_entries_from_two_threads():
    """cuda_ghmatece_ and cuda_send_gest_data_ at the same time, as the
    reference's two OpenMP sections call them, then GHMATECD + LINSOLVE
    through the seam; five rounds, each against the oracle."""
    s, d = meshgen.config_mesh("c1_240")
    d.kode[::9] = 0
    p = oracle.OracleProblem(s, d)
    _, ogd, _ = p.ghmatece()
    fr = 1.3
    odisp, otrac, ox = p.solve(fr, use_openblas=False)

    L = ctypes.CDLL(capi.LIB_PATH)
    P = capi.ptr
    bi = lambda v: ctypes.byref(ctypes.c_int(v))  # noqa: E731
    bd = lambda v: ctypes.byref(ctypes.c_double(v))  # noqa: E731
    gi, ome = host.gauleg(s.npg)
    cone = capi.i32(s.cone_fortran())
    cxm, cym, czm = (capi.f64(a) for a in s.centroids())
    etas = host.normvec(s.cone, s.cx, s.cy, s.cz)
    cx, cy, cz = capi.f64(s.cx), capi.f64(s.cy), capi.f64(s.cz)
    c = host.static_consts(s.ge, s.rnu)
    zge, zcs, zcp = host.material(s.ge, s.rnu, d.dam, d.rho)
    cz_ = lambda z: capi.f64([z.real, z.imag])  # noqa: E731
    gest = capi.f64(ogd)
    nn = 3 * s.nbe
    for rnd in range(5):
        L.send_shared_data_to_gpu_(P(cx), P(cy), P(cz), P(cxm), P(cym), P(czm), P(etas),
                                   P(capi.f64(gi)), P(capi.f64(ome)), P(cone), bi(s.np),
                                   bi(s.npg), bi(s.n), bi(s.nbe))
        status = ctypes.c_int(-1)
        hbuf = np.zeros(9 * s.nbe)
        go = threading.Barrier(2)
        errors = []

        def section_h():
            try:
                go.wait()
                L.cuda_ghmatece_(bi(s.nbe), bi(s.npg), bi(s.n), bi(s.np), bd(c[2]), bd(c[3]),
                                 bd(0.0), P(hbuf), ctypes.byref(status))
            except Exception as e:  # pragma: no cover - reported below
                errors.append(e)

        def section_g():
            try:
                go.wait()
                L.cuda_send_gest_data_(bi(s.nbe), P(gest))
            except Exception as e:  # pragma: no cover
                errors.append(e)

        th = [threading.Thread(target=section_h), threading.Thread(target=section_g)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert not errors and status.value == 0
        zdfi = capi.c128(d.bc)
        kode = capi.i32(d.kode)
        L.send_dyn_data_gpu_(bi(s.nbe), P(zdfi), P(kode))
        zfi = np.zeros(nn, dtype=np.complex128)
        zh = np.zeros(1, dtype=np.complex128)
        status.value = -1
        L.cuda_ghmatecd_(bi(s.nbe), bi(s.npg), bi(s.n), bi(s.np), P(cz_(zge)), P(cz_(zcs)),
                         P(cz_(zcp)), bd(c[0]), bd(c[1]), bd(c[2]), bd(c[3]), bd(fr), P(hbuf),
                         P(gest), P(zfi), P(zh), P(kode), bi(1), ctypes.byref(status))
        assert status.value == 0
        L.cuda_linsolve_(bi(nn), bi(s.n), P(zh), P(zfi))
        L.deallocate_shared_gpu_data_()
        assert rel(zfi, ox) < TOL, f"round {rnd}"
