"""Interior points on the device (bem_interior, cuda_interec1_): INTEREC's
displacements (src/Interec.for:81-135 with NONSINGD) and stresses
(src/Interec.for:186-285 with SIGMAEC, src/Sigmaec.for:9-212) against the
oracle's restatement on the same boundary solution, and the reference's own
known-answer files reproduced with every number computed on the GPU."""
import ctypes
import os

import numpy as np
import pytest

import oracle
import refcheck
import refmetrics
from bem_mececcs_b200 import capi, formats, host, meshgen
from bem_mececcs_b200.solver import BemSolver
from gpu_util import rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _points(l, seed=7):
    rng = np.random.default_rng(seed)
    return (rng.uniform(-4.0, 4.0, l), rng.uniform(-4.0, 4.0, l), rng.uniform(-2.0, -0.3, l))


def _solved(name="c1_240", fr=1.25, kode_zero_every=0):
    s, d = meshgen.config_mesh(name)
    if kode_zero_every:
        d.kode[::kode_zero_every] = 0
    sol = BemSolver(s)
    sol.ghmatece()
    sol.set_bc(d.kode, d.bc, d.dam, d.rho)
    disp, trac = sol.solve_frequency(fr)
    return s, d, sol, disp, trac


def test_interior_matches_oracle():
    fr = 1.25
    s, d, sol, disp, trac = _solved(fr=fr, kode_zero_every=5)
    cxi, cyi, czi = _points(9)
    zdsol, zssol = sol.interior(fr, disp, trac, cxi, cyi, czi)
    d.l, d.cxi, d.cyi, d.czi = 9, cxi, cyi, czi
    p = oracle.OracleProblem(s, d)
    ozd, ozs = p.interior(fr, disp, trac)
    assert rel(zdsol, ozd) < TOL
    assert refmetrics.zdsol(zdsol, ozd)[2]  # ASSERT_ZDSOL
    assert rel(zssol, ozs) < TOL
    # without stresses: the same displacements
    zd2, zs2 = sol.interior(fr, disp, trac, cxi, cyi, czi, stresses=False)
    assert zs2 is None and np.array_equal(zd2, zdsol)
    sol.ctx.close()


def test_interec1_seam_matches_native():
    """cuda_interec1_ after the seam's own sequence (src/Interec.for:59-67
    un-swap on the host, then the call at src/Interec.for:142-164)."""
    s, d = meshgen.config_mesh("c1_240")
    d.kode[::7] = 0
    fr = 0.8
    L = ctypes.CDLL(capi.LIB_PATH)
    P = capi.ptr
    bi = lambda v: ctypes.byref(ctypes.c_int(v))  # noqa: E731
    bd = lambda v: ctypes.byref(ctypes.c_double(v))  # noqa: E731
    gi, ome = host.gauleg(s.npg)
    cone = capi.i32(s.cone_fortran())
    cxm, cym, czm = (capi.f64(a) for a in s.centroids())
    etas = host.normvec(s.cone, s.cx, s.cy, s.cz)
    cx, cy, cz = capi.f64(s.cx), capi.f64(s.cy), capi.f64(s.cz)
    L.send_shared_data_to_gpu_(P(cx), P(cy), P(cz), P(cxm), P(cym), P(czm), P(etas),
                               P(capi.f64(gi)), P(capi.f64(ome)), P(cone), bi(s.np), bi(s.npg),
                               bi(s.n), bi(s.nbe))
    c = host.static_consts(s.ge, s.rnu)
    status = ctypes.c_int(-1)
    hbuf = np.zeros(9 * s.nbe)
    L.cuda_ghmatece_(bi(s.nbe), bi(s.npg), bi(s.n), bi(s.np), bd(c[2]), bd(c[3]), bd(0.0), P(hbuf),
                     ctypes.byref(status))
    p = oracle.OracleProblem(s, d)
    _, ogd, _ = p.ghmatece()
    L.cuda_send_gest_data_(bi(s.nbe), P(capi.f64(ogd)))
    zdfi = capi.c128(d.bc)
    kode = capi.i32(d.kode)
    L.send_dyn_data_gpu_(bi(s.nbe), P(zdfi), P(kode))
    zge, zcs, zcp = host.material(s.ge, s.rnu, d.dam, d.rho)
    cz_ = lambda z: capi.f64([z.real, z.imag])  # noqa: E731
    nn = 3 * s.nbe
    zfi = np.zeros(nn, dtype=np.complex128)
    zh = np.zeros(1, dtype=np.complex128)
    L.cuda_ghmatecd_(bi(s.nbe), bi(s.npg), bi(s.n), bi(s.np), P(cz_(zge)), P(cz_(zcs)), P(cz_(zcp)),
                     bd(c[0]), bd(c[1]), bd(c[2]), bd(c[3]), bd(fr), P(hbuf), P(capi.f64(ogd)),
                     P(zfi), P(zh), P(kode), bi(1), ctypes.byref(status))
    assert status.value == 0
    L.cuda_linsolve_(bi(nn), bi(s.n), P(zh), P(zfi))
    # INTEREC's un-swap on the host
    disp, trac = zfi.copy(), zdfi.copy()
    sw = d.kode == 0
    zch = disp[sw] * zge
    disp[sw] = trac[sw]
    trac[sw] = zch
    cxi, cyi, czi = (capi.f64(a) for a in _points(6, seed=11))
    zdsol = np.zeros(3 * 6, dtype=np.complex128)
    status.value = -1
    L.cuda_interec1_(bi(s.n), bi(s.nbe), bi(s.npg), bi(6), bi(s.np), P(cxi), P(cyi), P(czi),
                     P(cz_(zge)), P(cz_(zcs)), P(cz_(zcp)), bd(0.0), bd(0.0), bd(0.0), bd(0.0), bd(fr),
                     P(trac), P(disp), P(zdsol), ctypes.byref(status))
    assert status.value == 0
    L.deallocate_shared_gpu_data_()
    d.l, d.cxi, d.cyi, d.czi = 6, cxi, cyi, czi
    ozd, _ = oracle.OracleProblem(s, d).interior(fr, disp, trac)
    assert rel(zdsol, ozd) < TOL
    assert refmetrics.zdsol(zdsol, ozd)[2]  # ASSERT_ZDSOL


def _golden_on_gpu(golden_dir, stem, workdir):
    """dtester's errors of the all-GPU result (restated metric), and the
    reference's own checker run on it where oracle/_ref/dtester is built."""
    s = formats.read_static(os.path.join(golden_dir, f"ESOLO{stem}E_-5+5.DAT"))
    d = formats.read_dynamic(os.path.join(golden_dir, f"ESOLO{stem}D_-5+5.DAT"), s.nbe)
    sol = BemSolver(s)
    sol.ghmatece()
    sol.set_bc(d.kode, d.bc, d.dam, d.rho)
    fr = d.freqs[0]
    disp, trac = sol.solve_frequency(fr)
    zdsol, zssol = sol.interior(fr, disp, trac, d.cxi, d.cyi, d.czi)
    sol.ctx.close()
    mine = formats.Results(fr, disp.reshape(-1, 3), trac.reshape(-1, 3),
                           zdsol.reshape(-1, 3), zssol.reshape(-1, 9))
    gold_path = os.path.join(golden_dir, f"SSOLO{stem}D_-5+5.SOL")
    err = formats.dtester_errors(mine, formats.parse_results(gold_path)[0])
    ref = refcheck.check_run(s, d, mine, gold_path, workdir) if refcheck.available() else None
    return err, ref


def _check(err, ref):
    assert all(v <= 1e-3 for v in err.values()), err
    if ref is not None:
        rc, ref_err, file_err = ref
        assert rc == 0, ref_err
        for k, v in ref_err.items():
            assert v <= 1e-3 and v == pytest.approx(file_err[k], rel=1e-5, abs=1e-12), \
                (k, ref_err, file_err)


def test_golden_240_all_on_gpu(golden_dir, tmp_path):
    """src/tests.sh:38-50 with boundary AND interior results from the GPU."""
    _check(*_golden_on_gpu(golden_dir, "240", str(tmp_path)))


@pytest.mark.slow
def test_golden_2160_all_on_gpu(golden_dir, tmp_path):
    _check(*_golden_on_gpu(golden_dir, "2160", str(tmp_path)))
