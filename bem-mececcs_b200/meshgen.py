"""Seeded synthetic meshes in the reference's input formats.

Boundary surface: a planar surface z = 0 over [-5, 5] x [-5, 5] split into nx x ny four-node
quadrilateral constant elements.  Nodes are numbered row-major, element
(i, j) has corners (i,j), (i+1,j), (i+1,j+1), (i,j+1) counter-clockwise,
so that NORMVEC (src/Normvec.for:27-36) gives the normal +z.  Jitter moves
interior nodes only, uniformly by up to +-frac of the element's dx and dy,
so the domain boundary stays fixed; draws come from numpy's PCG64 with the
given seed (one (dx, dy) pair per node in node order, applied to interior
nodes).  `enclosed_grid` closes the surface into a box with non-collocated
enclosing elements, as the reference's own meshes do.  Boundary conditions: traction prescribed everywhere (KODE = 1),
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


def _quad_normal(p1, p2, p3):
    a, b = p2 - p1, p3 - p1
    return np.cross(a, b)


def enclosed_grid(nx: int, ny: int, *, jitter: float = 0.0, seed: int = 0, npg: int = 4,
                  ge: float = 1.0, rnu: float = 0.25, half: float = 5.0, depth: float = 2.5,
                  layers: int = 1) -> StaticInput:
    """`planar_grid` (the nx*ny boundary elements, normal +z) closed into a
    box by non-collocated enclosing elements, as the reference's own meshes
    are (src/ESOLO240E_-5+5.DAT: 100 boundary elements at z=0 plus a bottom
    and four walls with outward normals).  The enclosure lets the rigid-body
    row sum of the static H (src/Ghmatece.for:258-282) supply the free term;
    an open planar surface alone gives a singular H.  Bottom: the same x/y
    grid at z=-depth, normal -z; walls: `layers` element rows between the
    top perimeter (whose nodes are never jittered) and the bottom perimeter,
    outward normals.  Boundary elements come first (NBE = nx*ny)."""
    top = planar_grid(nx, ny, jitter=jitter, seed=seed, npg=npg, ge=ge, rnu=rnu, half=half)
    nt = (nx + 1) * (ny + 1)
    xs = np.linspace(-half, half, nx + 1)
    ys = np.linspace(-half, half, ny + 1)
    gx, gy = np.meshgrid(xs, ys)
    bx, by = gx.ravel(), gy.ravel()
    bz = np.full(nt, -depth)
    cx = [top.cx, bx]
    cy = [top.cy, by]
    cz = [top.cz, bz]
    # Perimeter loop of grid nodes (i, j), counter-clockwise seen from +z.
    per = ([(i, 0) for i in range(nx)] + [(nx, j) for j in range(ny)] +
           [(i, ny) for i in range(nx, 0, -1)] + [(0, j) for j in range(ny, 0, -1)])
    npr = len(per)
    node_top = lambda i, j: j * (nx + 1) + i + 1          # noqa: E731
    node_bot = lambda i, j: nt + j * (nx + 1) + i + 1     # noqa: E731
    # Intermediate wall layers.
    mids = []
    base = 2 * nt
    for lay in range(1, layers):
        z = -depth * lay / layers
        for (i, j) in per:
            cx.append(np.array([xs[i]]))
            cy.append(np.array([ys[j]]))
            cz.append(np.array([z]))
        mids.append(base + (lay - 1) * npr)
    cx, cy, cz = np.concatenate(cx), np.concatenate(cy), np.concatenate(cz)

    def wall_node(k, lay):
        i, j = per[k % npr]
        if lay == 0:
            return node_top(i, j)
        if lay == layers:
            return node_bot(i, j)
        return mids[lay - 1] + (k % npr) + 1

    pts = lambda q: [np.array([cx[v - 1], cy[v - 1], cz[v - 1]]) for v in q]  # noqa: E731
    cones = [top.cone]
    e_i, e_j = np.meshgrid(np.arange(nx), np.arange(ny))
    e_i, e_j = e_i.ravel(), e_j.ravel()
    bot = np.stack([node_bot(e_i, e_j), node_bot(e_i, e_j + 1), node_bot(e_i + 1, e_j + 1),
                    node_bot(e_i + 1, e_j)], axis=1)
    cones.append(bot.astype(np.int32))
    walls = []
    center = np.array([0.0, 0.0, -depth / 2])
    for k in range(npr):
        for lay in range(layers):
            q = [wall_node(k, lay), wall_node(k + 1, lay), wall_node(k + 1, lay + 1),
                 wall_node(k, lay + 1)]
            p = pts(q)
            nrm = _quad_normal(p[0], p[1], p[2])
            mid = sum(p) / 4
            if np.dot(nrm, mid - center) < 0:
                q = [q[0], q[3], q[2], q[1]]
            walls.append(q)
    cones.append(np.array(walls, dtype=np.int32))
    cone = np.concatenate(cones).astype(np.int32)
    title = (f"ENCLOSED {nx}x{ny} z=0 [-{half},{half}]^2 depth={depth} layers={layers} "
             f"jitter={jitter} seed={seed}")
    return StaticInput(title, cone.shape[0], nx * ny, cx.size, npg, ge, rnu, cx, cy, cz, cone)


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
    """The named synthetic workloads: (static input, dynamic input).

    Each is the planar boundary grid of its name (2160 elements = 48x45,
    n = 3*2160 = 6480 complex unknowns) closed by an enclosure of
    non-collocated elements (`enclosed_grid`, depth 2.5, 4 wall layers)."""
    enc = dict(depth=2.5, layers=4)
    if name == "c1_240":      # 16x15, no jitter, omega = 1
        m = enclosed_grid(16, 15, **enc)
        return m, traction_patch(m, freqs=(1.0,))
    if name == "c2_2160":     # 48x45, +-10% jitter, seed 0, omega = 2
        m = enclosed_grid(48, 45, jitter=0.10, seed=0, **enc)
        return m, traction_patch(m, freqs=(2.0,))
    if name == "c3_2160":     # precision form, seed 1
        m = enclosed_grid(48, 45, jitter=0.10, seed=1, **enc)
        return m, traction_patch(m, freqs=(0.5, 2.0, 8.0))
    if name == "c3_8640":     # precision form, seed 2
        m = enclosed_grid(96, 90, jitter=0.10, seed=2, **enc)
        return m, traction_patch(m, freqs=(0.5, 2.0, 8.0))
    raise KeyError(name)


def sweep_frequencies(count: int = 128, lo: float = 0.1, hi: float = 10.0,
                      seed: int = 3) -> np.ndarray:
    """The frequency sweep: omega log-uniform in [lo, hi], PCG64(seed)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))
