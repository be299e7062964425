"""driver.run_case on the GPU: the reference's ESOLO240 case from its input
files to its output files (src/tests.sh:38-53), every number computed by
libbem_b200.so.  The static output must be the shipped file byte for byte;
the dynamic output must pass the reference's check (src/dtester.c, EPS 1e-3),
by the restated metric and, where oracle/_ref/dtester was built, by the
reference's own checker on the written file."""
import os

import numpy as np
import pytest

import refcheck
from bem_mececcs_b200 import driver, formats

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_reference_case_through_the_driver(tmp_path, golden_dir, form):
    """Both forms of the driver: plain (one frequency at a time in FP64, what
    the reference does) and mixed (the lockstep sweep, FP32 LU on tensor
    cores + FP64 refinement) on the reference's NPG = 8 known-answer mesh."""
    ein = os.path.join(golden_dir, "ESOLO240E_-5+5.DAT")
    din = os.path.join(golden_dir, "ESOLO240D_-5+5.DAT")
    eout, dout = str(tmp_path / "SSOLO240E.DAT"), str(tmp_path / "SSOLO240D.DAT")
    res = driver.run_case(ein, din, eout, dout, form=form, device=0)
    assert len(res) == 1
    with open(os.path.join(golden_dir, "SSOLO240E_-5+5.SOL"), "rb") as fh:
        assert open(eout, "rb").read() == fh.read()
    gold_path = os.path.join(golden_dir, "SSOLO240D_-5+5.SOL")
    mine = formats.parse_results(dout)
    assert len(mine) == 1
    err = formats.dtester_errors(mine[0], formats.parse_results(gold_path)[0])
    assert all(np.isfinite(v) and v <= 1e-3 for v in err.values()), err
    if refcheck.available():
        rc, ref_err = refcheck.run(dout, gold_path)
        assert rc == 0, ref_err
