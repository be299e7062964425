"""The drop-in seam, called in the order and with the by-reference argument
convention of the reference's Fortran driver built with -DUSE_GPU:
src/Main.for:130 send_shared_data_to_gpu, src/Ghmatece.for:205,240
cuda_ghmatece + cuda_send_gest_data (GEST_SINGULAR computed on the host),
src/Main.for:162 send_dyn_data_gpu, src/Ghmatecd.for:198 cuda_ghmatecd
(fast_singular = 1), src/Linsolve.for:55 cuda_linsolve, src/Main.for:231
deallocate_shared_gpu_data."""
import ctypes

import numpy as np
import pytest

import oracle
from bem_mececcs_b200 import capi, host, meshgen
from gpu_util import rel

pytestmark = pytest.mark.gpu


def byref_int(v):
    return ctypes.byref(ctypes.c_int(v))


def byref_dbl(v):
    return ctypes.byref(ctypes.c_double(v))


def test_fortran_seam_sequence():
    s, d = meshgen.config_mesh("c1_240")
    d.kode[::7] = 0  # a few displacement-prescribed entries
    p = oracle.OracleProblem(s, d)
    ohd, ogd, _ = p.ghmatece()
    fr = 1.25
    odisp, otrac, ox = p.solve(fr, use_openblas=False)

    L = ctypes.CDLL(capi.LIB_PATH)
    P = capi.ptr
    gi, ome = host.gauleg(s.npg)
    cone = capi.i32(s.cone_fortran())
    cxm, cym, czm = (capi.f64(a) for a in s.centroids())
    etas = host.normvec(s.cone, s.cx, s.cy, s.cz)
    cx, cy, cz = capi.f64(s.cx), capi.f64(s.cy), capi.f64(s.cz)
    L.send_shared_data_to_gpu_(P(cx), P(cy), P(cz), P(cxm), P(cym), P(czm), P(etas),
                               P(capi.f64(gi)), P(capi.f64(ome)), P(cone), byref_int(s.np),
                               byref_int(s.npg), byref_int(s.n), byref_int(s.nbe))
    c = host.static_consts(s.ge, s.rnu)
    status = ctypes.c_int(-1)
    hbuf = np.zeros(9 * s.nbe)
    L.cuda_ghmatece_(byref_int(s.nbe), byref_int(s.npg), byref_int(s.n), byref_int(s.np),
                     byref_dbl(c[2]), byref_dbl(c[3]), byref_dbl(0.0), P(hbuf), ctypes.byref(status))
    assert status.value == 0
    L.cuda_send_gest_data_(byref_int(s.nbe), P(capi.f64(ogd)))  # host GEST_SINGULAR
    zdfi = capi.c128(d.bc)
    kode = capi.i32(d.kode)
    L.send_dyn_data_gpu_(byref_int(s.nbe), P(zdfi), P(kode))
    zge, zcs, zcp = host.material(s.ge, s.rnu, d.dam, d.rho)
    cz_ = lambda z: capi.f64([z.real, z.imag])  # noqa: E731
    nn = 3 * s.nbe
    zfi = np.zeros(nn, dtype=np.complex128)
    zh = np.zeros(1, dtype=np.complex128)
    status.value = -1
    L.cuda_ghmatecd_(byref_int(s.nbe), byref_int(s.npg), byref_int(s.n), byref_int(s.np),
                     P(cz_(zge)), P(cz_(zcs)), P(cz_(zcp)), byref_dbl(c[0]), byref_dbl(c[1]),
                     byref_dbl(c[2]), byref_dbl(c[3]), byref_dbl(fr), P(hbuf), P(capi.f64(ogd)),
                     P(zfi), P(zh), P(kode), byref_int(1), ctypes.byref(status))
    assert status.value == 0
    L.cuda_linsolve_(byref_int(nn), byref_int(s.n), P(zh), P(zfi))
    assert rel(zfi, ox) < 1e-10
    L.deallocate_shared_gpu_data_()
