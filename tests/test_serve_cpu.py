"""The serving workload generator and grid rounding (host logic, no GPU)."""
import numpy as np

from bem_mececcs_b200 import serve


def test_grid_for_is_close_and_square_ish():
    for e in (240, 241, 600, 1700, 2160, 5000, 12000):
        nx, ny = serve.grid_for(e)
        assert nx >= ny and nx * 9 <= ny * 10
        assert abs(nx * ny - e) <= max(nx, ny)


def test_workload_shape_and_determinism():
    w = serve.serving_workload(count=2000)
    assert len(w) == 2000
    t = np.array([r.t for r in w])
    assert np.all(np.diff(t) > 0)
    assert abs(2000 / t[-1] - 50.0) < 5.0           # mean rate 50/s
    frac = np.mean([r.rhs_only for r in w])
    assert abs(frac - 0.3) < 0.04
    sizes = np.array([r.grid[0] * r.grid[1] for r in w if not r.rhs_only])
    assert sizes.min() >= 200 and sizes.max() <= 12500
    # log-uniform: the median element count near sqrt(240 * 12000)
    assert 1000 < np.median(sizes) < 2800
    fr = np.array([r.fr for r in w])
    assert fr.min() >= 0.1 and fr.max() <= 10.0
    w2 = serve.serving_workload(count=2000)
    assert [(r.t, r.grid, r.fr, r.patch) for r in w] == [(r.t, r.grid, r.fr, r.patch) for r in w2]


def test_rhs_only_requests_reuse_an_earlier_problem():
    w = serve.serving_workload(count=300)
    first = {}
    for r in w:
        if not r.rhs_only:
            first[r.key] = r
        else:
            f = first[r.key]
            assert (r.grid, r.seed, r.fr, r.material) == (f.grid, f.seed, f.fr, f.material)
            assert r.patch != f.patch


def test_request_bc_patch():
    r = serve.Request(0.0, (16, 15), 3, 1.0, (1.0, 0.25, 0.01, 1.0), (0.0, 0.0, 1.0))
    m = serve.request_mesh(r)
    bc, kode = serve.request_bc(m, r)
    assert bc.shape == (3 * m.nbe,) and np.all(kode == 1)
    assert np.all(bc[0::3] == 0) and np.all(bc[1::3] == 0) and bc[2::3].sum() > 0
