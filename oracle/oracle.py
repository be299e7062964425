"""ctypes front end of the CPU FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the benchmark's
CPU-baseline leg use it as the checker.  The product path never imports it.

`OracleProblem` runs the reference's per-mesh and per-frequency pipeline
(src/Main.for:108-194) on the CPU: GAULEG, NORMVEC, GHMATECE, GHMATECD,
BOUNDARY_CONDITIONS, ZGEMV, ZGESV, INTEREC, and returns every intermediate.
The LU either runs the oracle's own restated ZGESV (small systems) or the
OpenBLAS ZGESV bundled with scipy, the LAPACK routine the reference links
(src/Linsolve.for:94-100, OpenBLAS 0.2.20 in the reference's deploy.sh).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_d = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_c = np.ctypeslib.ndpointer(dtype=np.complex128, flags="C_CONTIGUOUS")
_i = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_int, _dbl = ctypes.c_int, ctypes.c_double


def build() -> str:
    path = os.path.join(_HERE, "liboracle.so")
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return path


_BOUND: dict = {}

# The reference builds its CPU path with these (src/Makefile:17-18); the
# timing variant of the oracle uses them, the parity build does not.
REFERENCE_CFLAGS = ["-march=native", "-Ofast", "-funroll-loops", "-fopenmp"]


def timing_lib(outdir: str):
    """Compiles bem_oracle.c with the reference's CPU flags into outdir (on
    the machine that will run it: -march=native).  Returns (path, "") or,
    when that fails, (None, the compiler's complaint).  For timing only:
    -Ofast gives up the parity build's bit-for-bit arithmetic."""
    out = os.path.join(outdir, "liboracle_ofast.so")
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    try:
        r = subprocess.run([cc, *REFERENCE_CFLAGS, "-fPIC", "-std=c11", "-shared", "-o", out,
                            os.path.join(_HERE, "bem_oracle.c"), "-lm"],
                           capture_output=True, text=True, timeout=300)
    except (OSError, subprocess.TimeoutExpired) as e:
        return None, str(e)
    if r.returncode != 0:
        return None, (r.stderr.strip().splitlines() or ["compiler failed"])[-1]
    return out, ""


def lib(path: str | None = None):
    """The oracle's ctypes library: the parity build (liboracle.so) unless
    `path` names another build of bem_oracle.c."""
    global _LIB
    if path is not None:
        if path not in _BOUND:
            _BOUND[path] = _bind(ctypes.CDLL(path))
        return _BOUND[path]
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = _bind(ctypes.CDLL(path))
    return _LIB


def _bind(L):
    L.orc_gauleg.argtypes = [_int, _d, _d]
    L.orc_normvec.argtypes = [_int, _i, _d, _d, _d, _d]
    L.orc_centroids.argtypes = [_int, _i, _d, _d, _d, _d, _d, _d]
    L.orc_material.argtypes = [_dbl, _dbl, _dbl, _dbl, _d, _d, _d]
    L.orc_static_consts.argtypes = [_dbl, _dbl, _d]
    geo = [_int, _int, _int, _int, _i, _d, _d, _d]
    L.orc_ghmatece.argtypes = geo + [_d, _d, _d, _d, _d, _d, _dbl, _dbl, _d, _d,
                                     ctypes.c_void_p]
    L.orc_ghmatecd.argtypes = geo + [_d, _d, _d, _d, _d, _d, _d, _d, _d, _d, _dbl,
                                     _d, _d, _c, _c]
    L.orc_ghmatecd_cols.argtypes = geo + [_d, _d, _d, _d, _d, _d, _d, _d, _d, _d, _dbl,
                                          _d, _d, _int, _int, _c, _c]
    L.orc_boundary_conditions.argtypes = [_int, _c, _c, _i, _d]
    L.orc_zgemv.argtypes = [_int, _c, _c, _c]
    L.orc_zgesv.argtypes = [_int, _c, _i, _c]
    L.orc_unswap.argtypes = [_int, _i, _d, _c, _c]
    L.orc_interior_disp.argtypes = geo + [_d, _d, _d, _int, _d, _d, _d, _d, _d, _d,
                                          _dbl, _c, _c, _c]
    L.orc_interior_stress.argtypes = geo + [_d, _d, _d, _int, _d, _d, _d, _d, _d,
                                            _d, _dbl, _dbl, _c, _c, _c]
    L.orc_solfund.argtypes = [_d, _d, _d, _d, _d, _d, _dbl, _c, _c]
    L.orc_static_solve.argtypes = geo + [_d, _d, _d, _d, _d, _d, _dbl, _dbl, _i, _d, _d, _d,
                                         ctypes.c_void_p, ctypes.c_void_p]
    return L


def gauleg(npg: int):
    gi, ome = np.zeros(npg), np.zeros(npg)
    lib().orc_gauleg(npg, gi, ome)
    return gi, ome


def material(ge, rnu, dam, rho):
    zge, zcs, zcp = np.zeros(2), np.zeros(2), np.zeros(2)
    lib().orc_material(ge, rnu, dam, rho, zge, zcs, zcp)
    return zge, zcs, zcp


def static_consts(rmu, rnu):
    c = np.zeros(4)
    lib().orc_static_consts(rmu, rnu, c)
    return c


def zgesv(a: np.ndarray, b: np.ndarray, *, use_openblas: bool | None = None):
    """Solves A x = b for one right-hand side (column-major A as (n,n) F-order
    or its flat copy).  Returns x; a copy of A is factored."""
    n = b.shape[0]
    if use_openblas is None:
        use_openblas = n > 1500
    if use_openblas:
        from scipy.linalg import lapack
        af = np.array(a.reshape(n, n, order="F") if a.ndim == 1 else a, order="F",
                      dtype=np.complex128, copy=True)
        _, _, x, info = lapack.zgesv(af, b.astype(np.complex128).copy(),
                                     overwrite_a=True, overwrite_b=True)
        if info != 0:
            raise np.linalg.LinAlgError(f"ZGESV info={info}")
        return np.asarray(x).ravel()
    flat = np.ascontiguousarray((a.reshape(n, n, order="F") if a.ndim == 1 else a)
                                .ravel(order="F")).astype(np.complex128)
    x = b.astype(np.complex128).copy()
    piv = np.zeros(n, dtype=np.int32)
    if lib().orc_zgesv(n, flat, piv, x) != 0:
        raise np.linalg.LinAlgError("singular matrix")
    return x


class OracleProblem:
    """One mesh with its dynamic input, set up as src/Main.for:108-158 does."""

    def __init__(self, static, dynamic, lib_path: str | None = None):
        """lib_path: another build of bem_oracle.c (timing_lib) instead of
        the parity build."""
        self.s, self.d = static, dynamic
        self._lib = lib(lib_path)
        s = static
        self.cone = s.cone_fortran()
        self.cx = np.ascontiguousarray(s.cx, dtype=np.float64)
        self.cy = np.ascontiguousarray(s.cy, dtype=np.float64)
        self.cz = np.ascontiguousarray(s.cz, dtype=np.float64)
        self.gi, self.ome = gauleg(s.npg)
        self.etas = np.zeros(3 * s.n)
        self._lib.orc_normvec(s.n, self.cone, self.cx, self.cy, self.cz, self.etas)
        self.cxm, self.cym, self.czm = (np.zeros(s.n) for _ in range(3))
        self._lib.orc_centroids(s.n, self.cone, self.cx, self.cy, self.cz,
                            self.cxm, self.cym, self.czm)
        self.c = static_consts(s.ge, s.rnu)
        self.zge, self.zcs, self.zcp = material(s.ge, s.rnu, dynamic.dam, dynamic.rho)
        self.nn = 3 * s.nbe
        self.hestdiag = self.gestdiag = None

    def _geo(self):
        s = self.s
        return (s.n, s.nbe, s.np, s.npg, self.cone, self.cx, self.cy, self.cz)

    def ghmatece(self, want_hest: bool = False):
        s = self.s
        self.hestdiag = np.zeros(9 * s.nbe)
        self.gestdiag = np.zeros(9 * s.nbe)
        hest = np.zeros(9 * s.nbe * s.n) if want_hest else None
        st = self._lib.orc_ghmatece(*self._geo(), self.cxm, self.cym, self.czm, self.etas,
                                self.gi, self.ome, s.ge, s.rnu, self.hestdiag,
                                self.gestdiag,
                                hest.ctypes.data_as(ctypes.c_void_p) if hest is not None
                                else None)
        if st != 0:
            raise RuntimeError(f"GHMATECE status {st}")
        return self.hestdiag, self.gestdiag, hest

    def ghmatecd(self, fr: float):
        """Pre-swap ZH, ZG as flat column-major complex arrays."""
        if self.hestdiag is None:
            self.ghmatece()
        nn = self.nn
        zh = np.zeros(nn * nn, dtype=np.complex128)
        zg = np.zeros(nn * nn, dtype=np.complex128)
        st = self._lib.orc_ghmatecd(*self._geo(), self.cxm, self.cym, self.czm, self.etas,
                                self.gi, self.ome, self.c, self.zge, self.zcs, self.zcp,
                                float(fr), self.hestdiag, self.gestdiag, zh, zg)
        if st != 0:
            raise RuntimeError(f"GHMATECD status {st}")
        return zh, zg

    def ghmatecd_cols(self, fr: float, jlo: int, jhi: int, zh=None, zg=None):
        """GHMATECD restricted to element columns jlo..jhi-1 (timing samples)."""
        if self.hestdiag is None:
            self.ghmatece()
        nn = self.nn
        zh = np.zeros(nn * nn, dtype=np.complex128) if zh is None else zh
        zg = np.zeros(nn * nn, dtype=np.complex128) if zg is None else zg
        st = self._lib.orc_ghmatecd_cols(*self._geo(), self.cxm, self.cym, self.czm, self.etas,
                                     self.gi, self.ome, self.c, self.zge, self.zcs, self.zcp,
                                     float(fr), self.hestdiag, self.gestdiag, int(jlo), int(jhi),
                                     zh, zg)
        if st != 0:
            raise RuntimeError(f"GHMATECD status {st}")
        return zh, zg

    def static_solve(self, want_matrices: bool = False):
        """EXTENSION (no reference counterpart): the static boundary solve,
        orc_static_solve.  Returns (disp, trac[, h, g]) with the real BC
        values of the dynamic input (its real parts) and its KODE."""
        s, nn = self.s, self.nn
        kode = np.ascontiguousarray(self.d.kode, dtype=np.int32)
        dfi = np.ascontiguousarray(np.real(self.d.bc), dtype=np.float64)
        disp = np.zeros(nn)
        trac = np.zeros(nn)
        h = np.zeros(nn * nn) if want_matrices else None
        g = np.zeros(nn * nn) if want_matrices else None
        hp = h.ctypes.data_as(ctypes.c_void_p) if want_matrices else None
        gp = g.ctypes.data_as(ctypes.c_void_p) if want_matrices else None
        st = self._lib.orc_static_solve(*self._geo(), self.cxm, self.cym, self.czm, self.etas,
                                    self.gi, self.ome, float(s.ge), float(s.rnu), kode, dfi,
                                    disp, trac, hp, gp)
        if st != 0:
            raise RuntimeError(f"static solve status {st}")
        return (disp, trac, h, g) if want_matrices else (disp, trac)

    def system(self, fr: float, zdfi=None):
        """ZH after the boundary-condition swap and ZFI = ZG * ZDFI
        (src/Ghmatecd.for:168-181).  Returns (zh, zfi, zh_pre, zg_pre)."""
        zh, zg = self.ghmatecd(fr)
        zh0, zg0 = zh.copy(), zg.copy()
        kode = np.ascontiguousarray(self.d.kode, dtype=np.int32)
        self._lib.orc_boundary_conditions(self.nn, zh, zg, kode, self.zge)
        if zdfi is None:
            zdfi = self.d.bc.astype(np.complex128)
        zfi = np.zeros(self.nn, dtype=np.complex128)
        self._lib.orc_zgemv(self.nn, zg, np.ascontiguousarray(zdfi, dtype=np.complex128), zfi)
        return zh, zfi, zh0, zg0

    def solve(self, fr: float, *, use_openblas: bool | None = None, zdfi=None):
        """One frequency: LINSOLVE then the INTEREC un-swap.  Returns
        (boundary displacements, tractions, raw solution)."""
        zh, zfi, _, _ = self.system(fr, zdfi)
        x = zgesv(zh, zfi, use_openblas=use_openblas)
        disp = x.copy()
        tr = (self.d.bc.astype(np.complex128) if zdfi is None else
              np.asarray(zdfi, dtype=np.complex128)).copy()
        self._lib.orc_unswap(self.nn, np.ascontiguousarray(self.d.kode, dtype=np.int32),
                         self.zge, disp, tr)
        return disp, tr, x

    def interior(self, fr: float, zfi, zdfi):
        s, d = self.s, self.d
        zdsol = np.zeros(3 * d.l, dtype=np.complex128)
        zssol = np.zeros(9 * d.l, dtype=np.complex128)
        if d.l <= 0:
            return zdsol, zssol
        pts = [np.ascontiguousarray(a, dtype=np.float64) for a in (d.cxi, d.cyi, d.czi)]
        st = self._lib.orc_interior_disp(*self._geo(), self.etas, self.gi, self.ome, d.l,
                                     *pts, self.zge, self.zcs, self.zcp, float(fr),
                                     np.ascontiguousarray(zfi), np.ascontiguousarray(zdfi),
                                     zdsol)
        st |= self._lib.orc_interior_stress(*self._geo(), self.etas, self.gi, self.ome, d.l,
                                        *pts, self.zge, self.zcs, self.zcp, d.rho,
                                        float(fr), np.ascontiguousarray(zfi),
                                        np.ascontiguousarray(zdfi), zssol)
        if st != 0:
            raise RuntimeError(f"INTEREC status {st}")
        return zdsol, zssol
