"""The static boundary solve (bem_static_solve), an extension with no
reference counterpart (the reference keeps only the static diagonals): GPU
against the oracle's restatement (orc_static_solve) at 1e-10."""
import numpy as np
import pytest

import oracle
from bem_mececcs_b200 import meshgen
from bem_mececcs_b200.solver import BemSolver
from gpu_util import rel

pytestmark = pytest.mark.gpu


def _check(name, kode_zero_every):
    s, d = meshgen.config_mesh(name)
    if kode_zero_every:
        d.kode[::kode_zero_every] = 0
        d.bc[::kode_zero_every] = 0.01  # a small prescribed displacement there
    od, ot = oracle.OracleProblem(s, d).static_solve()
    sol = BemSolver(s)
    sol.ghmatece()
    disp, trac = sol.static_solve(d.kode, np.real(d.bc))
    sol.ctx.close()
    assert rel(disp, od) < 1e-10 and rel(trac, ot) < 1e-10


def test_static_solve_240():
    _check("c1_240", 0)


def test_static_solve_240_mixed_kode():
    _check("c1_240", 7)


@pytest.mark.slow
def test_static_solve_2160():
    _check("c2_2160", 0)
