"""The reference's in-process GPU-vs-CPU checks (built with -DTEST_CUDA),
restated: each returns (measured value, tolerance, passed) for a result of
ours against the oracle's, with the reference's metric and tolerance.  The
GPU tests apply them beside their own much tighter relative bounds, so that
they read like the reference's own tests."""
import numpy as np


def _check(value, eps):
    value = float(value)
    return value, eps, bool(value <= eps)


def ghmatece_h_g(hd, hd_ref, gd, gd_ref, nbe):
    """ASSERT_GHMATECE_H_G (src/Ghmatece.for:325-393): per element, the sum of
    |difference| over the 3x3 block of HESTdiag (and of GESTdiag); the max
    over elements must stay <= 1e-5 for both.  Returns the worse of the two."""
    h = np.abs(np.asarray(hd).reshape(nbe, 9) - np.asarray(hd_ref).reshape(nbe, 9)).sum(axis=1).max()
    g = np.abs(np.asarray(gd).reshape(nbe, 9) - np.asarray(gd_ref).reshape(nbe, 9)).sum(axis=1).max()
    return _check(max(h, g), 1.0e-5)


def ghmatecd_zh_zfi(zh, zh_ref, zfi, zfi_ref, nbe):
    """ASSERT_GHMATECD_ZH_ZFI (src/Ghmatecd.for:336-405): the max over columns
    of the column 1-norm of the ZH difference, and the max |difference| of
    ZFI, each <= 1.5e-6 NBE.  zh, zh_ref: (3 NBE, 3 NBE) column-major, flat or
    2-D.  (The reference loops over 3 N columns of a 3 NBE-column array; only
    the 3 NBE that exist are compared here.)"""
    nn = 3 * nbe
    a = np.asarray(zh).reshape(nn, nn, order="F") if np.ndim(zh) == 1 else np.asarray(zh)
    b = np.asarray(zh_ref).reshape(nn, nn, order="F") if np.ndim(zh_ref) == 1 else np.asarray(zh_ref)
    col = np.abs(a - b).sum(axis=0).max()
    rhs = np.abs(np.asarray(zfi) - np.asarray(zfi_ref)).max()
    return _check(max(col, rhs), 1.5e-6 * nbe)


def zfi(x, x_ref):
    """ASSERT_ZFI (src/Linsolve.for:112-141): max |difference| of the
    solution <= 1.2e-6."""
    return _check(np.abs(np.asarray(x) - np.asarray(x_ref)).max(), 1.2e-6)


def zdsol(z, z_ref):
    """ASSERT_ZDSOL (src/Interec.for:290-316): max |difference| of the
    interior displacements <= 1e-6."""
    return _check(np.abs(np.asarray(z) - np.asarray(z_ref)).max(), 1.0e-6)
