"""The batching form for meshes of uneven size (bem_batch_solve): problems of
24..600 elements with random Poisson ratio and damping, solved in padded
lockstep classes, against each problem solved alone (plain FP64 path:
1e-10; mixed form: 1e-8, the precision target)."""
import numpy as np
import pytest

from bem_mececcs_b200 import capi, meshgen, serve
from bem_mececcs_b200.solver import BemSolver, batch_solve, unswap_host
from gpu_util import rel

pytestmark = pytest.mark.gpu


def _problems(count, seed=9):
    rng = np.random.Generator(np.random.PCG64(seed))
    probs = []
    for k in range(count):
        nx, ny = serve.grid_for(int(rng.integers(24, 601)))
        nu = float(rng.uniform(0.15, 0.35))
        dam = float(rng.uniform(0.005, 0.05))
        m = meshgen.enclosed_grid(nx, ny, jitter=0.10, seed=int(rng.integers(1 << 30)), rnu=nu,
                                  depth=2.5, layers=4)
        d = meshgen.traction_patch(m, dam=dam, radius=float(rng.uniform(1.0, 3.0)))
        sol = BemSolver(m)
        sol.ghmatece()
        sol.set_bc(d.kode, d.bc, dam, 1.0)
        probs.append((sol, float(rng.uniform(0.1, 10.0)), d))
    return probs


@pytest.mark.parametrize("form,tol", [("plain", 1e-10), ("mixed", 1e-8)])
def test_batch_uneven_matches_alone(form, tol):
    probs = _problems(20)
    driver = capi.Context(0)
    xs, corr = batch_solve(driver, [(p[0], p[1]) for p in probs], form=form, refine=3)
    driver.close()
    for (sol, fr, d), x in zip(probs, xs):
        disp, trac = unswap_host(x, d.kode, d.bc, sol.material[0])
        da, ta = sol.solve_frequency(fr)
        assert rel(disp, da) < tol and rel(trac, ta) < tol, (sol.nn, fr)
    for p in probs:
        p[0].ctx.close()


def test_batch_equal_sizes_single_and_reuse():
    """Classes without padding (members of one size), a batch of one, and a
    second call on the same driver (its buffers reused, then grown): each
    result equals the problem solved alone."""
    meshes = [meshgen.enclosed_grid(8, 7, jitter=0.10, seed=s, depth=2.5, layers=4) for s in (1, 2, 3)]
    probs = []
    for k, m in enumerate(meshes):
        d = meshgen.traction_patch(m, radius=2.0)
        sol = BemSolver(m)
        sol.ghmatece()
        sol.set_bc(d.kode, d.bc, d.dam, d.rho)
        probs.append((sol, 0.7 + 1.3 * k, d))
    assert len({p[0].nn for p in probs}) == 1
    extra = _problems(3, seed=4)
    driver = capi.Context(0)
    for form, tol in (("plain", 1e-10), ("mixed", 1e-8)):
        for sub in (probs[:1], probs, probs + extra):
            xs, _ = batch_solve(driver, [(p[0], p[1]) for p in sub], form=form, refine=3)
            for (sol, fr, d), x in zip(sub, xs):
                disp, trac = unswap_host(x, d.kode, d.bc, sol.material[0])
                da, ta = sol.solve_frequency(fr)
                assert rel(disp, da) < tol and rel(trac, ta) < tol, (form, sol.nn, fr)
    driver.close()
    for p in probs + extra:
        p[0].ctx.close()
