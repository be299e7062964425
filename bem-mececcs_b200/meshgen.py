"""Seeded synthetic meshes in the reference's input formats.

A planar surface z = 0 over [-5, 5] x [-5, 5] split into nx x ny four-node
quadrilateral constant elements.  Nodes are numbered row-major, element
(i, j) has corners (i,j), (i+1,j), (i+1,j+1), (i,j+1) counter-clockwise,
so that NORMVEC (src/Normvec.for:27-36) gives the normal +z.  Jitter moves
interior nodes only, uniformly by up to +-frac of the element's dx and dy,
so the domain boundary stays fixed; draws come from numpy's PCG64 with the
given seed (one (dx, dy) pair per node in node order, applied to interior
nodes).  Boundary conditions: traction prescribed everywhere (KODE = 1),
unit vertical traction on elements whose centroid radius is below
`patch_radius`, zero elsewhere; no interior points.
"""
from __future__ import annotations

import numpy as np

from .formats import DynamicInput, StaticInput


def planar_grid(nx: int, ny: int, *, jitter: float = 0.0, seed: int = 0,
                npg: int = 4, ge: float = 1.0, rnu: float = 0.25,
                half: float = 5.0) -> StaticInput:
    xs = np.linspace(-half, half, nx + 1)
    ys = np.linspace(-half, half, ny + 1)
    gx, gy = np.meshgrid(xs, ys)  # (ny+1, nx+1), row-major nodes
    cx = gx.ravel().copy()
    cy = gy.ravel().copy()
    if jitter:
        rng = np.random.Generator(np.random.PCG64(seed))
        d = rng.uniform(-jitter, jitter, size=(cx.size, 2))
        ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1))
        interior = ((ii > 0) & (ii < nx) & (jj > 0) & (jj < ny)).ravel()
        dx, dy = 2 * half / nx, 2 * half / ny
        cx[interior] += d[interior, 0] * dx
        cy[interior] += d[interior, 1] * dy
    cz = np.zeros_like(cx)
    e_i, e_j = np.meshgrid(np.arange(nx), np.arange(ny))
    e_i, e_j = e_i.ravel(), e_j.ravel()
    node = lambda i, j: j * (nx + 1) + i + 1  # noqa: E731  (1-based)
    cone = np.stack([node(e_i, e_j), node(e_i + 1, e_j), node(e_i + 1, e_j + 1),
                     node(e_i, e_j + 1)], axis=1).astype(np.int32)
    n = nx * ny
    title = f"PLANAR {nx}x{ny} z=0 [-{half},{half}]^2 jitter={jitter} seed={seed}"
    return StaticInput(title, n, n, cx.size, npg, ge, rnu, cx, cy, cz, cone)


def traction_patch(mesh: StaticInput, *, radius: float = 1.0, dam: float = 0.01,
                   rho: float = 1.0, freqs=(1.0,), center=(0.0, 0.0),
                   value: float = 1.0) -> DynamicInput:
    cxm, cym, _ = mesh.centroids()
    r = np.hypot(cxm[: mesh.nbe] - center[0], cym[: mesh.nbe] - center[1])
    kode = np.ones(3 * mesh.nbe, dtype=np.int32)
    bc = np.zeros(3 * mesh.nbe)
    bc[2::3] = np.where(r < radius, value, 0.0)
    freqs = np.asarray(freqs, dtype=float)
    z = np.zeros(0)
    return DynamicInput("UNIT VERTICAL TRACTION PATCH", 0, freqs.size, dam, rho,
                        freqs, kode, bc, z, z.copy(), z.copy())


def config_mesh(name: str) -> tuple:
    """The named synthetic workloads: (static input, dynamic input)."""
    if name == "c1_240":      # 16x15, no jitter, omega = 1
        m = planar_grid(16, 15)
        return m, traction_patch(m, freqs=(1.0,))
    if name == "c2_2160":     # 48x45, +-10% jitter, seed 0, omega = 2
        m = planar_grid(48, 45, jitter=0.10, seed=0)
        return m, traction_patch(m, freqs=(2.0,))
    if name == "c3_2160":     # precision form, seed 1
        m = planar_grid(48, 45, jitter=0.10, seed=1)
        return m, traction_patch(m, freqs=(0.5, 2.0, 8.0))
    if name == "c3_8640":     # precision form, seed 2
        m = planar_grid(96, 90, jitter=0.10, seed=2)
        return m, traction_patch(m, freqs=(0.5, 2.0, 8.0))
    raise KeyError(name)


def sweep_frequencies(count: int = 128, lo: float = 0.1, hi: float = 10.0,
                      seed: int = 3) -> np.ndarray:
    """The frequency sweep: omega log-uniform in [lo, hi], PCG64(seed)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))
