"""The GPU on two meshes of the reference's own benchmark (src/bench.sh:3,
fixtures from malhas.zip): E510, a soil trench of 510 boundary and 5
enclosing elements, and Esoil_1600 (1600 + 5); NPG = 8, nu = 0.3, no damping,
omega = 1, L = 76 interior points.  A second geometry class after the planar
ESOLO meshes: a trench with walls and corners.

Every stage of the path against the FP64 oracle on the same input files, at
the plain path's 1e-10: the static diagonals (HESTdiag, GESTdiag), the
swapped system and right-hand side (GHMATECD), the solution (LINSOLVE), the
un-swapped boundary displacements and tractions (INTEREC), and the interior
displacements and stresses.  The mixed form's solution on the same system is
held to the 1e-8 target against the oracle's."""
import os

import numpy as np
import pytest

import oracle
from bem_mececcs_b200 import formats
from bem_mececcs_b200.solver import BemSolver
from gpu_util import rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _read(golden_dir, name):
    s = formats.read_static(os.path.join(golden_dir, f"{name}e.dat"))
    d = formats.read_dynamic(os.path.join(golden_dir, f"{name}d.dat"), s.nbe)
    return s, d


@pytest.mark.parametrize("name", ["E510", pytest.param("Esoil_1600", marks=pytest.mark.slow)])
def test_benchmark_mesh_against_oracle(golden_dir, name):
    s, d = _read(golden_dir, name)
    fr = float(d.freqs[0])
    # the oracle: GHMATECE, GHMATECD + swap + ZGEMV, ZGESV, un-swap, INTEREC
    p = oracle.OracleProblem(s, d)
    ohd, ogd, _ = p.ghmatece()
    ozh, ozfi, _, _ = p.system(fr)
    ox = oracle.zgesv(ozh, ozfi, use_openblas=True)
    odisp, otrac = ox.copy(), d.bc.astype(np.complex128).copy()
    p._lib.orc_unswap(p.nn, np.ascontiguousarray(d.kode, dtype=np.int32), p.zge, odisp, otrac)
    ozd, ozs = p.interior(fr, odisp, otrac)

    sol = BemSolver(s)
    hd, gd = sol.ghmatece(compute_gest=True)
    assert rel(hd, ohd) < 1e-12
    assert rel(gd, ogd) < 1e-12
    sol.set_bc(d.kode, d.bc, d.dam, d.rho)
    sol.ghmatecd(fr)
    zh, zfi = sol.get_system()
    assert rel(zh, ozh) < TOL
    assert rel(zfi, ozfi) < TOL
    x = sol.linsolve()
    assert rel(x, ox) < TOL
    disp, trac = sol.interec()
    assert rel(disp, odisp) < TOL
    assert rel(trac, otrac) < TOL
    zdsol, zssol = sol.interior(fr, disp, trac, d.cxi, d.cyi, d.czi)
    assert rel(zdsol, ozd) < TOL
    assert rel(zssol, ozs) < TOL
    xm, corr = sol.sweep([fr], form="mixed", batch=1, refine=3)
    err = rel(xm[0], ox)
    print(name, "n", sol.nn, "mixed vs oracle", err, "last correction", float(corr[0]))
    assert err < 1e-8
    sol.close()
