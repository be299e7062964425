"""The reference's own golden-file checker on the oracle's output.

src/tests.sh:38-117 checks a run by compiling src/dtester.c and running it on
the run's output file against the shipped SSOLO*D_-5+5.SOL.  oracle/Makefile
(`make -C oracle ref`) compiles that checker from the reference tree into
oracle/_ref/dtester; these tests write the oracle's solution of ESOLO240 and
ESOLO2160 as the reference's output file (formats.write_dynamic_output) and
require that

- the oracle's result block, printed to the golden file's 4 digits, is the
  shipped one byte for byte, and the reference's checker accepts it (exit
  status 0, every error zero),
- the four errors it prints equal formats.dtester_errors, the restatement the
  GPU parity tests use, to the printed precision,
- a mistake planted in the oracle's output (one displacement moved by 2e-3) is
  rejected by both.

Skipped where neither the built checker nor the reference tree is present.
"""
import os

import numpy as np
import pytest

import oracle
import refcheck
from bem_mececcs_b200 import formats

EPS = 1.0e-3  # src/dtester.c:24


@pytest.fixture(scope="module")
def dtester():
    if not refcheck.build():
        pytest.skip("the reference's checker is not built and its source is absent")
    return refcheck.DTESTER


def _oracle_results(golden_dir, tag):
    s = formats.read_static(os.path.join(golden_dir, f"ESOLO{tag}E_-5+5.DAT"))
    d = formats.read_dynamic(os.path.join(golden_dir, f"ESOLO{tag}D_-5+5.DAT"), s.nbe)
    p = oracle.OracleProblem(s, d)
    p.ghmatece()
    fr = d.freqs[0]
    disp, tr, _ = p.solve(fr)
    zdsol, zssol = p.interior(fr, disp, tr)
    return s, d, formats.Results(fr, disp.reshape(-1, 3), tr.reshape(-1, 3),
                                 zdsol.reshape(-1, 3), zssol.reshape(-1, 9))


@pytest.mark.parametrize("tag", ["240", pytest.param("2160", marks=pytest.mark.slow)])
def test_reference_checker_accepts_the_oracle(tmp_path, golden_dir, dtester, tag):
    gold_path = os.path.join(golden_dir, f"SSOLO{tag}D_-5+5.SOL")
    s, d, res = _oracle_results(golden_dir, tag)
    ours = str(tmp_path / f"ours{tag}.SOL")
    refcheck.write(ours, s, d, res)

    rc, ref_err = refcheck.run(ours, gold_path)
    assert rc == 0, ref_err
    # printed to the golden file's 4 digits, the oracle's result block is the
    # shipped one byte for byte, so every error the checker prints is zero
    assert formats.format_results(res) == refcheck.result_block(gold_path)
    assert all(v == 0.0 for v in ref_err.values()), ref_err
    # the restated metric on the same two files
    mine = formats.parse_results(ours)[0]
    gold = formats.parse_results(gold_path)[0]
    err = formats.dtester_errors(mine, gold)
    for k in ref_err:
        assert err[k] <= EPS
        assert err[k] == pytest.approx(ref_err[k], rel=1e-5, abs=1e-12), k


def test_reference_checker_rejects_a_planted_mistake(tmp_path, golden_dir, dtester):
    gold_path = os.path.join(golden_dir, "SSOLO240D_-5+5.SOL")
    s, d, res = _oracle_results(golden_dir, "240")
    res.disp = res.disp.copy()
    res.disp[17, 1] += 2.0e-3
    ours = str(tmp_path / "planted.SOL")
    refcheck.write(ours, s, d, res)

    rc, ref_err = refcheck.run(ours, gold_path)
    assert rc == 1 and ref_err["disp"] > EPS
    err = formats.dtester_errors(formats.parse_results(ours)[0],
                                 formats.parse_results(gold_path)[0])
    assert err["disp"] > EPS
    assert err["disp"] == pytest.approx(ref_err["disp"], rel=1e-5)
    # the other three quantities are untouched and still pass
    for k in ("traction", "idisp", "sigma"):
        assert ref_err[k] <= EPS and err[k] == pytest.approx(ref_err[k], rel=1e-5, abs=1e-12)


def test_reference_checker_on_the_golden_file_itself(golden_dir, dtester):
    for tag in ("240", "2160"):
        g = os.path.join(golden_dir, f"SSOLO{tag}D_-5+5.SOL")
        rc, ref_err = refcheck.run(g, g)
        assert rc == 0 and all(v == 0.0 for v in ref_err.values())
        assert np.all(np.isfinite(formats.parse_results(g)[0].sigma))
