"""CPU-only checks of the C-ABI library and of the host-side setup."""
import ctypes

import numpy as np
import pytest

import oracle
from bem_mececcs_b200 import capi, host, meshgen


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(capi.LIB_PATH)
    names = capi.header_functions()
    assert "cuda_ghmatecd_" in names and "bem_linsolve" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_seam_names_match_gfortran_mangling():
    # The reference's Fortran calls these (src/Main.for:130,162,231;
    # src/Ghmatece.for:205,240; src/Ghmatecd.for:198; src/Linsolve.for:55).
    seam = ["send_shared_data_to_gpu_", "send_dyn_data_gpu_", "cuda_ghmatece_",
            "cuda_send_gest_data_", "cuda_ghmatecd_", "cuda_linsolve_",
            "deallocate_shared_gpu_data_"]
    lib = ctypes.CDLL(capi.LIB_PATH)
    for name in seam:
        assert hasattr(lib, name), name


@pytest.mark.parametrize("npg", [1, 2, 3, 4, 6, 8])
def test_host_gauleg_matches_oracle(npg):
    gi, ome = host.gauleg(npg)
    ogi, oome = oracle.gauleg(npg)
    assert np.array_equal(gi, ogi) and np.array_equal(ome, oome)


def test_host_setup_matches_oracle():
    s, d = meshgen.config_mesh("c2_2160")
    p = oracle.OracleProblem(s, d)
    etas = host.normvec(s.cone, s.cx, s.cy, s.cz)
    assert np.max(np.abs(etas - p.etas)) < 1e-15
    cxm, cym, czm = s.centroids()
    assert np.array_equal(cxm, p.cxm) and np.array_equal(cym, p.cym)
    assert np.allclose(host.static_consts(s.ge, s.rnu), p.c, rtol=1e-15, atol=0)
    zge, zcs, zcp = host.material(s.ge, s.rnu, d.dam, d.rho)
    assert abs(zge - complex(*p.zge)) < 1e-15
    assert abs(zcs - complex(*p.zcs)) < 1e-15 and abs(zcp - complex(*p.zcp)) < 1e-14


def test_meshgen_configs():
    s, d = meshgen.config_mesh("c1_240")
    # 240 boundary elements + bottom 240 + walls 2*(16+15)*4.
    assert (s.nbe, s.n, s.npg) == (240, 240 + 240 + 248, 4)
    assert d.kode.min() == 1 and d.bc[2::3].sum() > 0
    s2, _ = meshgen.config_mesh("c2_2160")
    assert s2.nbe == 2160 and s2.n == 2160 * 2 + 2 * (48 + 45) * 4
    # Jitter keeps the domain boundary fixed and moves interior nodes.
    assert s2.cx.min() == -5.0 and s2.cx.max() == 5.0
    s0 = meshgen.enclosed_grid(48, 45, depth=2.5, layers=4)
    assert not np.array_equal(s0.cx, s2.cx)
    assert np.max(np.abs(s0.cx - s2.cx)) <= 0.1 * 10 / 48 + 1e-12


def test_enclosure_normals_point_outward():
    s, _ = meshgen.config_mesh("c1_240")
    et = host.normvec(s.cone, s.cx, s.cy, s.cz).reshape(-1, 3)
    cxm, cym, czm = s.centroids()
    assert np.allclose(et[: s.nbe], [0, 0, 1])  # boundary surface: +z
    mid = np.stack([cxm, cym, czm + 1.25], 1)   # box centre at z = -1.25
    assert np.all(np.sum(et[s.nbe:] * mid[s.nbe:], axis=1) > 0)


def test_planar_mesh_alone_is_singular():
    """Why the synthetic meshes are enclosed: an open planar surface with
    N = NBE gives a singular H (no free term from the rigid-body sum)."""
    s = meshgen.planar_grid(6, 5)
    d = meshgen.traction_patch(s, radius=2.0)
    p = oracle.OracleProblem(s, d)
    p.ghmatece()
    zh, _, _, _ = p.system(1.0)
    sv = np.linalg.svd(zh.reshape(p.nn, p.nn, order="F"), compute_uv=False)
    assert sv[0] / sv[-1] > 1e12
    s = meshgen.enclosed_grid(6, 5, depth=2.5, layers=4)
    p = oracle.OracleProblem(s, meshgen.traction_patch(s, radius=2.0))
    p.ghmatece()
    zh, _, _, _ = p.system(1.0)
    sv = np.linalg.svd(zh.reshape(p.nn, p.nn, order="F"), compute_uv=False)
    assert sv[0] / sv[-1] < 100
