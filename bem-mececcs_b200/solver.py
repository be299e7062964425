"""The reference's per-mesh / per-frequency pipeline on the GPU.

`BemSolver` mirrors the reference driver (src/Main.for:108-194) and its
routines, each backed by the C-ABI of libbem_b200.so:

  ghmatece()   GHMATECE   (src/Ghmatece.for:9-256): HESTdiag, GESTdiag
  set_bc()     send_dyn_data_gpu_ (ZDFI = BC, KODE; src/Main.for:151-163)
  ghmatecd()   GHMATECD   (src/Ghmatecd.for:11-239): swapped ZH, ZFI = ZG*ZDFI
  linsolve()   LINSOLVE   (src/Linsolve.for:1-66): ZFI <- ZH^-1 ZFI
  interec()    INTEREC un-swap (src/Interec.for:59-67): displacements, tractions

Errors: a degenerate Jacobian raises BemError(BEM_ERR_DEGENERATE) where the
reference prints "Matriz Singular" / STOPs; a singular ZH raises
BemError(BEM_ERR_SINGULAR) where the reference's lu_assert exits.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import host
from .capi import (BEM_FAST_SINGULAR, BEM_FORM_MIXED, BEM_FORM_PLAIN, BEM_KEEP_PRESWAP, BemError,
                   Context, c128, f64, i32, ptr)


class BemSolver:
    def __init__(self, static, device: int = 0, ctx: Context | None = None):
        self.s = static
        self._own_ctx = ctx is None
        self.ctx = ctx or Context(device)
        s = static
        self.nn = 3 * s.nbe
        self.gi, self.ome = host.gauleg(s.npg)
        self.cone = i32(s.cone_fortran())
        self.cx, self.cy, self.cz = f64(s.cx), f64(s.cy), f64(s.cz)
        self.etas = host.normvec(s.cone, self.cx, self.cy, self.cz)
        self.cxm, self.cym, self.czm = (f64(a) for a in s.centroids())
        self.c = host.static_consts(s.ge, s.rnu)
        L = self.ctx.L
        self.ctx.check(L.bem_mesh_upload(self.ctx.h, s.n, s.nbe, s.np, s.npg, ptr(self.cone),
                                         ptr(self.cx), ptr(self.cy), ptr(self.cz), ptr(self.cxm),
                                         ptr(self.cym), ptr(self.czm), ptr(self.etas),
                                         ptr(f64(self.gi)), ptr(f64(self.ome))),
                       "bem_mesh_upload")
        self.kode = None
        self.zdfi = None
        self.material = None

    def close(self):
        """Frees the device state: the context, when this solver created it
        (a context passed in belongs to the caller)."""
        if self._own_ctx and self.ctx is not None:
            self.ctx.close()
        self.ctx = None if self._own_ctx else self.ctx

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False

    def ghmatece(self, compute_gest: bool = True):
        hd = np.zeros(9 * self.s.nbe)
        gd = np.zeros(9 * self.s.nbe)
        self.ctx.check(self.ctx.L.bem_ghmatece(self.ctx.h, ptr(f64(self.c)), int(compute_gest),
                                               ptr(hd), ptr(gd)), "bem_ghmatece")
        return hd, (gd if compute_gest else None)

    def static_h(self):
        out = np.zeros(9 * self.s.nbe * self.s.n)
        self.ctx.check(self.ctx.L.bem_static_h(self.ctx.h, ptr(f64(self.c)), ptr(out)),
                       "bem_static_h")
        return out

    def static_solve(self, kode, dfi):
        """Static boundary solve (bem_static_solve, an extension with no
        reference counterpart): real boundary displacements and tractions.
        Needs ghmatece() first."""
        nn = self.nn
        disp = np.zeros(nn)
        trac = np.zeros(nn)
        self.ctx.check(self.ctx.L.bem_static_solve(self.ctx.h, ptr(f64(self.c)), float(self.s.ge),
                                                   ptr(i32(kode)), ptr(f64(dfi)), ptr(disp), ptr(trac)),
                       "bem_static_solve")
        return disp, trac

    def set_gestdiag(self, gd):
        self.ctx.check(self.ctx.L.bem_set_gestdiag(self.ctx.h, ptr(f64(gd))), "bem_set_gestdiag")

    def set_bc(self, kode, zdfi, dam: float, rho: float):
        self.kode = i32(kode)
        self.zdfi = c128(zdfi)
        self.material = host.material(self.s.ge, self.s.rnu, dam, rho)
        self.rho = float(rho)
        self.ctx.check(self.ctx.L.bem_dyn_upload(self.ctx.h, ptr(self.zdfi), ptr(self.kode)),
                       "bem_dyn_upload")

    def ghmatecd(self, fr: float, *, keep_preswap: bool = False, fast_singular: bool = True):
        zge, zcs, zcp = self.material
        flags = (BEM_FAST_SINGULAR if fast_singular else 0) | (BEM_KEEP_PRESWAP if keep_preswap else 0)
        self.ctx.check(self.ctx.L.bem_ghmatecd(
            self.ctx.h, ptr(f64([zge.real, zge.imag])), ptr(f64([zcs.real, zcs.imag])),
            ptr(f64([zcp.real, zcp.imag])), ptr(f64(self.c)), float(fr), flags), "bem_ghmatecd")

    def get_system(self):
        zh = np.zeros(self.nn * self.nn, dtype=np.complex128)
        zfi = np.zeros(self.nn, dtype=np.complex128)
        self.ctx.check(self.ctx.L.bem_get_system(self.ctx.h, ptr(zh), ptr(zfi)), "bem_get_system")
        return zh, zfi

    def get_preswap(self):
        zh = np.zeros(self.nn * self.nn, dtype=np.complex128)
        zg = np.zeros(self.nn * self.nn, dtype=np.complex128)
        self.ctx.check(self.ctx.L.bem_get_preswap(self.ctx.h, ptr(zh), ptr(zg)), "bem_get_preswap")
        return zh, zg

    def linsolve(self):
        zfi = np.zeros(self.nn, dtype=np.complex128)
        self.ctx.check(self.ctx.L.bem_linsolve(self.ctx.h, ptr(zfi)), "bem_linsolve")
        return zfi

    def interec(self):
        disp = np.zeros(self.nn, dtype=np.complex128)
        trac = np.zeros(self.nn, dtype=np.complex128)
        self.ctx.check(self.ctx.L.bem_unswap(self.ctx.h, ptr(disp), ptr(trac)), "bem_unswap")
        return disp, trac

    def interior(self, fr: float, disp, trac, cxi, cyi, czi, *, rho: float | None = None,
                 stresses: bool = True):
        """INTEREC's interior part on the device (bem_interior): displacements
        zdsol (3L) and, with stresses, zssol (9L) at the points (cxi, cyi, czi)
        from the boundary displacements and tractions of the un-swap."""
        cxi, cyi, czi = f64(cxi), f64(cyi), f64(czi)
        l = int(cxi.size)
        zge, zcs, zcp = self.material
        if rho is None:
            rho = self.rho
        zdsol = np.zeros(3 * l, dtype=np.complex128)
        zssol = np.zeros(9 * l, dtype=np.complex128) if stresses else None
        self.ctx.check(self.ctx.L.bem_interior(
            self.ctx.h, ptr(f64([zge.real, zge.imag])), ptr(f64([zcs.real, zcs.imag])),
            ptr(f64([zcp.real, zcp.imag])), float(rho), float(fr), l, ptr(cxi), ptr(cyi), ptr(czi),
            ptr(c128(disp)), ptr(c128(trac)), ptr(zdsol), ptr(zssol)), "bem_interior")
        return zdsol, zssol

    def sweep(self, freqs, *, form: str = "mixed", batch: int = 8, refine: int = 3,
              want_x: bool = True, fallback_tol: float | None = None):
        """Frequency sweep on the resident mesh (bem_sweep).  Returns
        (x[nfreq, nn] raw solutions or None, last relative correction).

        fallback_tol (mixed form, refine > 0, x wanted): a problem whose last
        refinement correction is above it, or not finite, has not converged
        (refinement stalls when the FP32 factors are too far from the FP64
        matrix); it is solved again in the plain FP64 form and its index is
        listed in self.fallbacks.  Its correction is left as reported."""
        self.fallbacks = []
        x, corr = self._sweep_raw(freqs, form, batch, refine, want_x)
        if fallback_tol is None or form != "mixed" or not want_x or refine <= 0:
            return x, corr
        idx = [i for i, c in enumerate(corr) if not c <= fallback_tol]
        if idx:
            plain_batch = max(1, min(batch, self.sweep_batch_limit("plain")))
            xp, _ = self._sweep_raw(f64(freqs)[idx], "plain", plain_batch, refine, True)
            x[idx] = xp
            self.fallbacks = idx
        return x, corr

    def _sweep_raw(self, freqs, form, batch, refine, want_x):
        freqs = f64(freqs)
        nf = freqs.size
        zge, zcs, zcp = self.material
        x = np.zeros((nf, self.nn), dtype=np.complex128) if want_x else None
        corr = np.zeros(nf) if want_x else None
        fm = BEM_FORM_MIXED if form == "mixed" else BEM_FORM_PLAIN
        self.ctx.check(self.ctx.L.bem_sweep(
            self.ctx.h, ptr(f64([zge.real, zge.imag])), ptr(f64([zcs.real, zcs.imag])),
            ptr(f64([zcp.real, zcp.imag])), ptr(f64(self.c)), ptr(freqs), nf, fm, batch, refine,
            ptr(x), ptr(corr)), "bem_sweep")
        return x, corr

    def sweep_async(self, freqs, x_out, *, form: str = "mixed", batch: int = 8, refine: int = 3):
        """bem_sweep_async: enqueues the sweep and the copy of its raw
        solutions into x_out (complex128, len(freqs) x nn, page-locked for
        the copy to overlap) and returns at once.  x_out must stay alive and
        untouched until the context's stream has passed the copy (an event
        on that stream, or self.ctx.sync(), which also reports errors)."""
        freqs = f64(freqs)
        if x_out.dtype != np.complex128 or x_out.size < freqs.size * self.nn or not x_out.flags.c_contiguous:
            raise ValueError("x_out: contiguous complex128 with len(freqs) * nn entries")
        zge, zcs, zcp = self.material
        fm = BEM_FORM_MIXED if form == "mixed" else BEM_FORM_PLAIN
        self.ctx.check(self.ctx.L.bem_sweep_async(
            self.ctx.h, ptr(f64([zge.real, zge.imag])), ptr(f64([zcs.real, zcs.imag])),
            ptr(f64([zcp.real, zcp.imag])), ptr(f64(self.c)), ptr(freqs), freqs.size, fm, batch, refine,
            ptr(x_out)), "bem_sweep_async")

    def sweep_batch_limit(self, form: str = "mixed") -> int:
        """Largest lockstep batch bem_sweep uses for this mesh and form."""
        out = ctypes.c_int(0)
        fm = BEM_FORM_MIXED if form == "mixed" else BEM_FORM_PLAIN
        self.ctx.check(self.ctx.L.bem_sweep_batch_limit(self.ctx.h, fm, ctypes.byref(out)),
                       "bem_sweep_batch_limit")
        return int(out.value)

    def solve_frequency(self, fr: float):
        """GHMATECD + LINSOLVE + un-swap: boundary displacements and tractions."""
        self.ghmatecd(fr)
        self.linsolve()
        return self.interec()


def batch_solve(driver: Context, problems, *, form: str = "mixed", refine: int = 3):
    """bem_batch_solve: problems = [(BemSolver with ghmatece() and set_bc()
    done, omega), ...] of uneven sizes, solved in padded lockstep classes on
    the driver context.  Returns (list of raw solutions, corrections); the
    un-swapped (disp, trac) of problem p follow from `unswap_host`."""
    n = len(problems)
    ctxs = (ctypes.c_void_p * n)(*[p[0].ctx.h.value for p in problems])
    freqs = f64([p[1] for p in problems])
    zge = f64([[p[0].material[0].real, p[0].material[0].imag] for p in problems])
    zcs = f64([[p[0].material[1].real, p[0].material[1].imag] for p in problems])
    zcp = f64([[p[0].material[2].real, p[0].material[2].imag] for p in problems])
    c = f64([p[0].c for p in problems])
    xs = [np.zeros(p[0].nn, dtype=np.complex128) for p in problems]
    xptr = (ctypes.c_void_p * n)(*[x.ctypes.data for x in xs])
    corr = np.zeros(n)
    fm = BEM_FORM_MIXED if form == "mixed" else BEM_FORM_PLAIN
    driver.check(driver.L.bem_batch_solve(driver.h, n, ctxs, ptr(freqs), ptr(zge), ptr(zcs), ptr(zcp),
                                          ptr(c), fm, refine, xptr, ptr(corr)), "bem_batch_solve")
    return xs, corr


def unswap_host(x, kode, zdfi, zge):
    """Interec.for:59-67 on the host: (boundary displacements, tractions)."""
    x = np.asarray(x)
    kode = np.asarray(kode)
    zdfi = np.asarray(zdfi, dtype=np.complex128)
    disp = np.where(kode == 0, zdfi, x)
    trac = np.where(kode == 0, x * zge, zdfi)
    return disp, trac


def solve_dense(ctx: Context, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """ZGESV on the device for one right-hand side; a is (n, n)."""
    n = b.shape[0]
    af = c128(np.asarray(a).reshape(n, n).ravel(order="F"))
    x = np.zeros(n, dtype=np.complex128)
    ctx.check(ctx.L.bem_solve_dense(ctx.h, n, ptr(af), ptr(c128(b)), ptr(x)), "bem_solve_dense")
    return x


__all__ = ["BemSolver", "BemError", "solve_dense"]
