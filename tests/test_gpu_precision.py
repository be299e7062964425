"""The precision form on the configurations it is specified for: jittered
2160- and 8640-element meshes (n = 6480 and 25920) at omega in {0.5, 2, 8};
the mixed form (FP32 LU on tcgen05 + FP64 refinement) against the plain FP64
GPU path, which itself matches the FP64 oracle to 1e-10 (test_gpu_parity).
The per-result relative errors are printed (pytest -s) and bounded by the
1e-8 target."""
import numpy as np
import pytest

from bem_mececcs_b200 import meshgen
from bem_mececcs_b200.solver import BemSolver

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
def test_precision_8640():
    assert max(_errors("c3_8640", 1)) < 1e-8
