"""The serving form: ctypes wrapper of the library's request loop
(bem_server_*, include/bem_capi.h) and the seeded synthetic request stream
it is measured on.

The loop itself is native (csrc/serve.cu): requests are admitted by device
footprint as they arrive, run concurrently on their own streams, and solved
problems stay resident so that a new right-hand side for the same (mesh,
material, omega, KODE) reuses the factors.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import host, meshgen
from .capi import BEM_FORM_MIXED, BEM_FORM_PLAIN, BEM_OK, BemError, c128, f64, i32, lib, ptr


class Server:
    """One GPU's request loop (bem_server_create)."""

    def __init__(self, device: int = 0, budget_bytes: float = 160e9, form: str = "mixed",
                 refine: int = 3):
        L = lib()
        vp, ip, dp, P = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.POINTER
        L.bem_server_create.argtypes = [ip, dp, ip, ip, P(vp)]
        L.bem_server_destroy.argtypes = [vp]
        L.bem_server_add_mesh.argtypes = [vp, ip, ip, ip, ip] + [vp] * 10 + [P(ip)]
        L.bem_server_submit.argtypes = [vp, ip, vp, dp, vp, vp, P(ctypes.c_longlong)]
        L.bem_server_wait.argtypes = [vp, ctypes.c_longlong, dp, vp, vp, vp]
        L.bem_server_stats.argtypes = [vp, vp]
        L.bem_server_reset_stats.argtypes = [vp]
        self.L = L
        self.h = vp()
        fm = BEM_FORM_MIXED if form == "mixed" else BEM_FORM_PLAIN
        rc = L.bem_server_create(device, float(budget_bytes), fm, refine, ctypes.byref(self.h))
        if rc != BEM_OK:
            raise BemError(rc, "bem_server_create failed")
        self.nn = {}

    def add_mesh(self, s) -> int:
        """Registers a StaticInput; returns its mesh id."""
        gi, ome = host.gauleg(s.npg)
        cone = i32(s.cone_fortran())
        cx, cy, cz = f64(s.cx), f64(s.cy), f64(s.cz)
        cxm, cym, czm = (f64(a) for a in s.centroids())
        etas = host.normvec(s.cone, cx, cy, cz)
        mid = ctypes.c_int(-1)
        rc = self.L.bem_server_add_mesh(self.h, s.n, s.nbe, s.np, s.npg, ptr(cone), ptr(cx), ptr(cy),
                                        ptr(cz), ptr(cxm), ptr(cym), ptr(czm), ptr(etas),
                                        ptr(f64(gi)), ptr(f64(ome)), ctypes.byref(mid))
        if rc != BEM_OK:
            raise BemError(rc, "bem_server_add_mesh failed")
        self.nn[mid.value] = 3 * s.nbe
        return mid.value

    def submit(self, mesh_id: int, material, fr: float, bc, kode) -> int:
        """material = (GE, nu, damping, density)."""
        rid = ctypes.c_longlong(0)
        rc = self.L.bem_server_submit(self.h, mesh_id, ptr(f64(material)), float(fr), ptr(c128(bc)),
                                      ptr(i32(kode)), ctypes.byref(rid))
        if rc != BEM_OK:
            raise BemError(rc, "bem_server_submit failed")
        self._pending = getattr(self, "_pending", {})
        self._pending[rid.value] = self.nn[mesh_id]
        return rid.value

    def wait(self, rid: int, timeout: float = 300.0):
        """(disp, trac, info) of a request; raises BemError on its failure."""
        nn = self._pending[rid]
        disp = np.zeros(nn, dtype=np.complex128)
        trac = np.zeros(nn, dtype=np.complex128)
        info = np.zeros(4)
        rc = self.L.bem_server_wait(self.h, rid, float(timeout), ptr(disp), ptr(trac), ptr(info))
        if rc != BEM_OK:
            raise BemError(rc, f"request {rid}")
        del self._pending[rid]
        return disp, trac, {"latency_ms": float(info[0]), "queue_ms": float(info[1]),
                            "rhs_only": bool(info[2]), "bytes": int(info[3])}

    def stats(self) -> dict:
        out = np.zeros(10)
        self.L.bem_server_stats(self.h, ptr(out))
        keys = ["completed", "p50_ms", "p99_ms", "solves_per_s", "rhs_only", "evictions",
                "peak_bytes", "max_busy", "bytes_now", "budget"]
        return {k: float(v) for k, v in zip(keys, out)}

    def reset_stats(self):
        self.L.bem_server_reset_stats(self.h)

    def close(self):
        if self.h:
            self.L.bem_server_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# The serving workload: Poisson arrivals, mesh sizes log-uniform on
# rectangular jittered grids, omega uniform, a share of right-hand-side-only
# requests on problems seen before.  Everything is seeded (PCG64).
# ---------------------------------------------------------------------------

@dataclass
class Request:
    t: float                 # arrival time, seconds from the start
    grid: tuple              # (nx, ny) boundary elements
    seed: int                # jitter seed of the mesh
    fr: float
    material: tuple          # (GE, nu, damping, density)
    patch: tuple             # traction patch (cx, cy, radius)
    rhs_only: bool = False   # same mesh, omega and material as an earlier request
    key: int = field(default=0)  # index of the (mesh, omega) problem


def grid_for(elements: int) -> tuple:
    """The rectangular nx x ny grid (nx >= ny, aspect <= 10/9) closest to
    `elements` boundary elements."""
    best = None
    for ny in range(max(1, int(np.sqrt(elements * 0.9)) - 2), int(np.sqrt(elements)) + 3):
        for nx in (ny, int(round(elements / ny))):
            if nx < ny or nx * 9 > ny * 10:
                continue
            err = abs(nx * ny - elements)
            if best is None or err < best[0]:
                best = (err, nx, ny)
    return best[1], best[2]


def serving_workload(count: int = 2000, rate: float = 50.0, lo: int = 240, hi: int = 12000,
                     rhs_frac: float = 0.3, seed: int = 4,
                     material=(1.0, 0.25, 0.01, 1.0)) -> list:
    """The serving stream: `count` Poisson arrivals at `rate` per second;
    element counts log-uniform in [lo, hi] rounded to rectangular grids;
    omega uniform in [0.1, 10]; a fraction `rhs_frac` of the requests reuse
    the mesh, omega and material of an earlier request with a new random
    traction patch (unit vertical traction inside the patch)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = np.cumsum(rng.exponential(1.0 / rate, size=count))
    out, problems = [], []
    for i in range(count):
        patch = (float(rng.uniform(-3.0, 3.0)), float(rng.uniform(-3.0, 3.0)),
                 float(rng.uniform(0.5, 2.0)))
        if problems and rng.uniform() < rhs_frac:
            k = int(rng.integers(len(problems)))
            g, sd, fr = problems[k]
            out.append(Request(float(t[i]), g, sd, fr, tuple(material), patch, True, k))
        else:
            e = float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
            g = grid_for(int(round(e)))
            sd = int(rng.integers(1 << 30))
            fr = float(rng.uniform(0.1, 10.0))
            problems.append((g, sd, fr))
            out.append(Request(float(t[i]), g, sd, fr, tuple(material), patch, False,
                               len(problems) - 1))
    return out


def request_mesh(req: Request):
    """The enclosed, jittered mesh of a request (as the sweep's meshes)."""
    return meshgen.enclosed_grid(req.grid[0], req.grid[1], jitter=0.10, seed=req.seed,
                                 depth=2.5, layers=4)


def request_bc(mesh, req: Request):
    """(bc, kode): unit vertical traction on boundary elements inside the
    request's patch, traction prescribed everywhere (KODE = 1)."""
    cxm, cym, _ = mesh.centroids()
    r = np.hypot(cxm[: mesh.nbe] - req.patch[0], cym[: mesh.nbe] - req.patch[1])
    bc = np.zeros(3 * mesh.nbe, dtype=np.complex128)
    bc[2::3] = np.where(r < req.patch[2], 1.0, 0.0)
    return bc, np.ones(3 * mesh.nbe, dtype=np.int32)
