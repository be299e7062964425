"""bem_ghmatecd_noalloc: the GHMATECD assembly for callers that may not
allocate device memory after set-up (a serving process whose HBM is already
handed to its own pool, a loop that cannot take cudaFree's device-wide
synchronisation).  It writes into a buffer the caller owns and takes its
scratch from a fixed 8 MiB array in the library, so its output must equal
what bem_ghmatecd + bem_get_system give for the same frequency.

This file is named to be collected last: it also has to pass after every
other GPU test of the session has left its own state on the device.
"""
import ctypes

import numpy as np
import pytest

from bem_mececcs_b200 import capi, meshgen
from bem_mececcs_b200.solver import BemSolver
from gpu_util import rel

pytestmark = pytest.mark.gpu

TOL = 1e-10  # the plain FP64 parity tolerance of the GPU tests


def _cz(z):
    return capi.f64([z.real, z.imag])


def _call(sol, fr, buf_ptr, lda, flags=capi.BEM_FAST_SINGULAR):
    zge, zcs, zcp = sol.material
    return sol.ctx.L.bem_ghmatecd_noalloc(sol.ctx.h, capi.ptr(_cz(zge)), capi.ptr(_cz(zcs)),
                                          capi.ptr(_cz(zcp)), capi.ptr(capi.f64(sol.c)), float(fr),
                                          flags, ctypes.c_void_p(buf_ptr), lda)


@pytest.mark.parametrize("flags", [0, capi.BEM_FAST_SINGULAR])
def test_noalloc_matches_ghmatecd_two_calls_in_a_row(flags):
    torch = pytest.importorskip("torch")
    s, d = meshgen.config_mesh("c1_240")
    d.kode[::5] = 0  # displacement-prescribed entries: exercises the column swap
    sol = BemSolver(s)
    sol.ghmatece()
    sol.set_bc(d.kode, d.bc, d.dam, d.rho)
    nn = sol.nn
    freqs = (0.75, 2.5)
    want = []
    for fr in freqs:
        sol.ghmatecd(fr, fast_singular=bool(flags & capi.BEM_FAST_SINGULAR))
        want.append(sol.get_system())

    lda = nn + 3  # padded leading dimension, columns of lda complex128
    bufs = [torch.full((nn + 1, lda), float("nan"), dtype=torch.complex128, device="cuda:0")
            for _ in freqs]
    torch.cuda.synchronize()
    launches = sol.ctx.launches
    for fr, buf in zip(freqs, bufs):  # back to back: the second call reuses the scratch
        sol.ctx.check(_call(sol, fr, buf.data_ptr(), lda, flags), "bem_ghmatecd_noalloc")
    sol.ctx.check(sol.ctx.L.bem_sync(sol.ctx.h), "bem_sync")
    assert sol.ctx.launches - launches == 3 * len(freqs)

    for (zh, zfi), buf in zip(want, bufs):
        a = buf.cpu().numpy()  # row c of the array is column c of the system
        assert rel(a[:nn, :nn].reshape(-1), zh) < TOL
        assert rel(a[nn, :nn], zfi) < TOL
        assert np.isnan(a[:, nn:].real).all()  # rows nn..lda-1 of each column untouched
    sol.ctx.close()


def test_noalloc_rejects_mesh_beyond_scratch_limit():
    torch = pytest.importorskip("torch")
    # 42 x 42 elements at NPG = 8: 16 elements per column chunk, so the RHS
    # partials alone need ceil(1764/16) * 5292 * 16 bytes > 8 MiB.
    s = meshgen.planar_grid(42, 42, npg=8)
    d = meshgen.traction_patch(s)
    sol = BemSolver(s)
    sol.set_bc(d.kode, d.bc, d.dam, d.rho)
    buf = torch.empty((1, 2), dtype=torch.complex128, device="cuda:0")
    launches = sol.ctx.launches
    rc = _call(sol, 1.0, buf.data_ptr(), 3 * s.nbe, flags=0)
    assert rc == capi.BEM_ERR_ARG
    assert "fixed limit" in sol.ctx.L.bem_last_error(sol.ctx.h).decode()
    assert sol.ctx.launches == launches
    sol.ctx.close()


# The largest mesh each Gauss rule accepts and the first one it rejects.  The
# scratch is 18 nbe words for the diagonal blocks (rounded up to 16 words)
# plus ceil(nbe / jc) x 3 nbe words of RHS partials, jc = min(64, 1024 / npg^2)
# elements per column chunk, 16 bytes a word, against 8 MiB.
LIMITS = [(4, 3136, (56, 56), (3137, 1)),
          (6, 2128, (56, 38), (2129, 1)),
          (8, 1618, (809, 2), (1619, 1))]


@pytest.mark.parametrize("npg,nbe_max,grid_ok,grid_over", LIMITS,
                         ids=[f"npg{x[0]}" for x in LIMITS])
def test_noalloc_limit_boundary(npg, nbe_max, grid_ok, grid_over):
    """At the documented maximum the call runs and equals bem_ghmatecd; one
    element more is refused before any launch."""
    torch = pytest.importorskip("torch")
    assert grid_ok[0] * grid_ok[1] == nbe_max and grid_over[0] * grid_over[1] == nbe_max + 1
    s = meshgen.planar_grid(*grid_over, npg=npg)
    d = meshgen.traction_patch(s)
    sol = BemSolver(s)
    sol.set_bc(d.kode, d.bc, d.dam, d.rho)
    buf = torch.empty((1, 2), dtype=torch.complex128, device="cuda:0")
    launches = sol.ctx.launches
    assert _call(sol, 1.0, buf.data_ptr(), 3 * s.nbe, flags=0) == capi.BEM_ERR_ARG
    assert "fixed limit" in sol.ctx.L.bem_last_error(sol.ctx.h).decode()
    assert sol.ctx.launches == launches
    sol.ctx.close()

    s = meshgen.planar_grid(*grid_ok, npg=npg)
    d = meshgen.traction_patch(s, radius=3.0)  # reaches the centroids of every strip (|y| <= 2.5)
    assert np.abs(d.bc).sum() > 0
    sol = BemSolver(s)
    sol.set_bc(d.kode, d.bc, d.dam, d.rho)
    nn = sol.nn
    sol.ghmatecd(1.0, fast_singular=False)
    zh, zfi = sol.get_system()
    buf = torch.full((nn + 1, nn), float("nan"), dtype=torch.complex128, device="cuda:0")
    torch.cuda.synchronize()
    sol.ctx.check(_call(sol, 1.0, buf.data_ptr(), nn, flags=0), "bem_ghmatecd_noalloc")
    sol.ctx.check(sol.ctx.L.bem_sync(sol.ctx.h), "bem_sync")
    a = buf.cpu().numpy()
    del buf
    assert rel(a[:nn].reshape(-1), zh) < TOL
    assert rel(a[nn], zfi) < TOL
    sol.ctx.close()
