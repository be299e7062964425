"""The precision form on the configurations it is specified for: jittered
2160- and 8640-element meshes (n = 6480 and 25920) at omega in {0.5, 2, 8}.
On 2160 elements every result of both forms is checked against the FP64
oracle itself (boundary displacements and tractions after the un-swap:
mixed <= 1e-8, plain <= 1e-10).  On 8640 elements (the oracle would need
about 25 GB and minutes per omega) the mixed form is checked against the
plain FP64 GPU path, which matches the oracle wherever both run.  The
per-result relative errors are printed (pytest -s)."""
import numpy as np
import pytest

import oracle
from bem_mececcs_b200 import meshgen
from bem_mececcs_b200.solver import BemSolver, unswap_host
from gpu_util import rel

pytestmark = pytest.mark.gpu


def _errors(name, batch):
    s, d = meshgen.config_mesh(name)
    sol = BemSolver(s)
    sol.ghmatece()
    sol.set_bc(d.kode, d.bc.astype(np.complex128), d.dam, d.rho)
    xm, corr = sol.sweep(d.freqs, form="mixed", batch=batch, refine=3)
    xp, _ = sol.sweep(d.freqs, form="plain", batch=batch)
    sol.ctx.close()
    errs = [float(np.linalg.norm(xm[i] - xp[i]) / np.linalg.norm(xp[i])) for i in range(len(d.freqs))]
    print(name, "omega", list(d.freqs), "rel err mixed vs FP64", errs, "last correction", list(corr))
    return errs


def test_precision_2160():
    assert max(_errors("c3_2160", 3)) < 1e-8


@pytest.mark.slow
def test_precision_2160_against_oracle():
    s, d = meshgen.config_mesh("c3_2160")
    sol = BemSolver(s)
    sol.ghmatece()
    sol.set_bc(d.kode, d.bc.astype(np.complex128), d.dam, d.rho)
    xm, corr = sol.sweep(d.freqs, form="mixed", batch=3, refine=3)
    xp, _ = sol.sweep(d.freqs, form="plain", batch=3)
    zge = sol.material[0]
    sol.close()
    p = oracle.OracleProblem(s, d)
    p.ghmatece()
    for i, fr in enumerate(d.freqs):
        odisp, otrac, ox = p.solve(float(fr), use_openblas=True)
        for form, x, tol in (("mixed", xm[i], 1e-8), ("plain", xp[i], 1e-10)):
            disp, trac = unswap_host(x, d.kode, d.bc, zge)
            e = (rel(x, ox), rel(disp, odisp), rel(trac, otrac))
            print("c3_2160 omega", fr, form, "rel err vs oracle (x, disp, trac)", e,
                  "last correction", float(corr[i]))
            assert max(e) < tol, (fr, form, e)


@pytest.mark.slow
def test_precision_8640():
    assert max(_errors("c3_8640", 1)) < 1e-8
