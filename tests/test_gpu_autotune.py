"""Context options and the sweep autotuner: every switch setting gives the
same solutions (graph replay included), and the tuner's cache round-trips."""
import numpy as np
import pytest

from bem_mececcs_b200 import autotune, meshgen
from bem_mececcs_b200.solver import BemSolver
from gpu_util import rel

pytestmark = pytest.mark.gpu


def _solver(name="c1_240"):
    s, d = meshgen.config_mesh(name)
    sol = BemSolver(s)
    sol.ghmatece()
    sol.set_bc(d.kode, d.bc, d.dam, d.rho)
    return sol


def test_options_give_the_same_solutions():
    sol = _solver()
    freqs = meshgen.sweep_frequencies(14, seed=3)
    ref, _ = sol.sweep(freqs, form="mixed", batch=7, refine=3)
    # graphs: the second and later batches (and calls) replay a captured step
    again, _ = sol.sweep(freqs, form="mixed", batch=7, refine=3)
    assert np.array_equal(again, ref)
    for opt, val in (("graphs", False), ("lu_pairs", False), ("panel_calu", True), ("trsv_coop", False),
                     ("panel_push", False), ("trsv_inv", False), ("laswp_tc", False), ("lu_quads", False),
                     ("panel_async", False)):
        sol.ctx.set_option(opt, val)
        assert sol.ctx.get_option(opt) == val
        x, _ = sol.sweep(freqs, form="mixed", batch=7, refine=3)
        assert max(rel(x[i], ref[i]) for i in range(len(freqs))) < 1e-12, opt
        sol.ctx.set_option(opt, not val)
    sol.ctx.close()


def test_autotune_cache_roundtrip(tmp_path):
    sol = _solver()
    freqs = meshgen.sweep_frequencies(32, seed=3)
    path = str(tmp_path / "tune.json")
    best = autotune.tune_sweep(sol, freqs, form="mixed", steps=1, space={"graphs": (True, False)},
                               batches=[7, 4], cache_path=path)
    assert best["solves_per_s"] > 0 and len(best["candidates"]) == 4
    cfg = autotune.tuned(sol, "mixed", path)
    assert cfg["batch"] == best["batch"] and cfg["options"] == best["options"]
    sol.ctx.close()
