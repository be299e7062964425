"""Host-side setup of the reference's driver (src/Main.for:108-158).

Computed once per mesh / material on the CPU before the device is called,
exactly where the reference computes them: the Gauss-Legendre rule
(GAULEG, src/Gauleg.for:9-36), element normals (NORMVEC,
src/Normvec.for:4-39), collocation points (src/Inputece.for:100-102), the
static constants C1..C4 (src/Ghmatece.for:55-63) and the complex material
(src/Inputecd.for:58-60).
"""
from __future__ import annotations

import math

import numpy as np


def gauleg(npg: int):
    """GAULEG(-1, 1, GI, OME, NPG): Newton on the Legendre polynomial."""
    x = np.zeros(npg)
    w = np.zeros(npg)
    m = (npg + 1) // 2
    xm, xl = 0.0, 1.0
    for i in range(1, m + 1):
        z = math.cos(3.141592654 * (i - 0.25) / (npg + 0.5))
        while True:
            p1, p2 = 1.0, 0.0
            for j in range(1, npg + 1):
                p3 = p2
                p2 = p1
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j
            pp = npg * (z * p1 - p2) / (z * z - 1.0)
            z1 = z
            z = z1 - p1 / pp
            if abs(z - z1) <= 3.0e-14:
                break
        x[i - 1] = xm - xl * z
        x[npg - i] = xm + xl * z
        w[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp)
        w[npg - i] = w[i - 1]
    return x, w


def normvec(cone: np.ndarray, cx, cy, cz) -> np.ndarray:
    """ETAS(3,N) flattened column-major: unit (P2-P1)x(P3-P1)."""
    c = np.asarray(cone) - 1
    p1 = np.stack([cx[c[:, 0]], cy[c[:, 0]], cz[c[:, 0]]], 1)
    p2 = np.stack([cx[c[:, 1]], cy[c[:, 1]], cz[c[:, 1]]], 1)
    p3 = np.stack([cx[c[:, 2]], cy[c[:, 2]], cz[c[:, 2]]], 1)
    a, b = p2 - p1, p3 - p1
    nrm = np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1],
                    a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                    a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], 1)
    r = np.sqrt(np.sum(nrm * nrm, axis=1, keepdims=True))
    return np.ascontiguousarray((nrm / r).ravel())


def static_consts(rmu: float, rnu: float) -> np.ndarray:
    pi = 4.0 * math.atan(1.0)
    return np.array([1.0 / (16.0 * pi * rmu * (1.0 - rnu)), 3.0 - 4.0 * rnu,
                     -1.0 / (8.0 * pi * (1.0 - rnu)), 1.0 - 2.0 * rnu])


def material(ge: float, rnu: float, dam: float, rho: float):
    """ZGE, ZCS, ZCP as complex numbers."""
    zge = complex(ge, ge * 2.0 * dam)
    zcs = complex(np.sqrt(np.complex128(zge / rho)))
    zcp = zcs * math.sqrt((2.0 - 2.0 * rnu) / (1.0 - 2.0 * rnu))
    return zge, zcs, zcp
