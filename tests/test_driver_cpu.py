"""driver.run_case, the reference's main program over its four files
(src/Main.for:85-200), with an oracle-backed stand-in for the GPU solver.

The stand-in has BemSolver's interface and answers from the oracle, so the
driver's own work (reading, echoing, the frequency loop, the un-swap of the
mixed form, interior points, writing) is checked here on the CPU: on the
reference's ESOLO240 case both output files must be the shipped ones byte for
byte, and a multi-frequency case with prescribed displacements must give each
frequency the solution of its own system from the file's boundary conditions.
The GPU solver behind the same calls is checked in tests/test_gpu_driver.py.
"""
import os
import re
import types

import numpy as np
import pytest

import oracle
from bem_mececcs_b200 import driver, formats, host
from bem_mececcs_b200.solver import BemSolver


class OracleSolver:
    """BemSolver's interface, answered by the oracle (test only)."""

    def __init__(self, s, d):
        self.s, self.d = s, d
        self.p = oracle.OracleProblem(s, d)
        self.ctx = types.SimpleNamespace(close=lambda: None, sync=lambda: None)
        self.calls = []

    def ghmatece(self):
        self.calls.append("ghmatece")
        self.p.ghmatece()

    def set_bc(self, kode, zdfi, dam, rho):
        self.calls.append("set_bc")
        assert np.array_equal(kode, self.d.kode) and np.array_equal(zdfi, self.d.bc)
        self.material = host.material(self.s.ge, self.s.rnu, dam, rho)

    def ghmatecd(self, fr):
        self.calls.append(("solve", fr))
        self.fr = fr

    def linsolve(self):
        self.last = self.p.solve(self.fr, use_openblas=False)
        return self.last[2]

    def interec(self):
        return self.last[0], self.last[1]

    stall = ()  # frequencies whose mixed refinement the stand-in reports as stalled

    def sweep_batch_limit(self, form):
        return 7

    sweep = BemSolver.sweep  # the real fallback logic over the stand-in's raw sweep

    def _sweep_raw(self, freqs, form, batch, refine, want_x):
        freqs = [float(f) for f in freqs]
        self.calls.append(("sweep", tuple(freqs), form, batch))
        x = np.array([self.p.solve(f, use_openblas=False)[2] for f in freqs])
        corr = np.zeros(len(freqs))
        if form == "mixed":
            for i, f in enumerate(freqs):
                if f in self.stall:  # a stalled refinement: a wrong x, a large correction
                    x[i] *= 1.5
                    corr[i] = 1e-3
        return x, corr

    def interior(self, fr, disp, trac, cxi, cyi, czi):
        self.calls.append(("interior", fr))
        return self.p.interior(fr, disp, trac)


def _factory(d, made):
    def make(s, device):
        sol = OracleSolver(s, d)
        made.append(sol)
        return sol
    return make


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_reference_case_files_come_out_byte_identical(tmp_path, golden_dir, form):
    ein = os.path.join(golden_dir, "ESOLO240E_-5+5.DAT")
    din = os.path.join(golden_dir, "ESOLO240D_-5+5.DAT")
    s = formats.read_static(ein)
    d = formats.read_dynamic(din, s.nbe)
    made = []
    eout, dout = tmp_path / "SSOLO240E.DAT", tmp_path / "SSOLO240D.DAT"
    res = driver.run_case(ein, din, eout, dout, form=form, solver_factory=_factory(d, made))
    assert len(res) == 1 and res[0].freq == d.freqs[0]
    for out, gold in ((eout, "SSOLO240E_-5+5.SOL"), (dout, "SSOLO240D_-5+5.SOL")):
        with open(os.path.join(golden_dir, gold), "rb") as fh:
            assert out.read_bytes() == fh.read(), gold
    calls = made[0].calls
    assert calls[:2] == ["ghmatece", "set_bc"]
    if form == "mixed":
        assert calls[2] == ("sweep", (float(d.freqs[0]),), "mixed", 7)
    else:
        assert calls[2] == ("solve", float(d.freqs[0]))


def test_every_frequency_starts_from_the_file_boundary_conditions(tmp_path, golden_dir):
    """Three frequencies, a third of the components with prescribed
    displacement: each block is the solution of that frequency's own system
    from the file's BCs (the reference's in-place ZDFI update is not carried
    from one frequency to the next)."""
    ein = os.path.join(golden_dir, "ESOLO240E_-5+5.DAT")
    s = formats.read_static(ein)
    d = formats.read_dynamic(os.path.join(golden_dir, "ESOLO240D_-5+5.DAT"), s.nbe)
    rng = np.random.default_rng(8)
    d.freqs = np.array([0.5, 1.0, 2.25])
    d.nfr = 3
    d.kode = np.where(rng.random(d.kode.size) < 0.33, 0, 1).astype(np.int32)
    d.bc = np.where(d.kode == 0, 0.01 * rng.standard_normal(d.kode.size), d.bc)
    din = tmp_path / "d.dat"
    formats.write_dynamic(din, d)
    d2 = formats.read_dynamic(din, s.nbe)
    outs = {}
    for form in ("plain", "mixed"):
        made = []
        res = driver.run_case(ein, din, tmp_path / f"e_{form}", tmp_path / f"d_{form}", form=form,
                              solver_factory=_factory(d2, made))
        back = formats.parse_results(tmp_path / f"d_{form}")
        assert [b.freq for b in back] == pytest.approx([0.5, 1.0, 2.25])
        p = oracle.OracleProblem(s, d2)
        p.ghmatece()
        for r, fr in zip(res, (0.5, 1.0, 2.25)):
            disp, trac, _ = p.solve(fr, use_openblas=False)
            assert np.allclose(r.disp.ravel(), disp, rtol=0, atol=1e-13 * np.abs(disp).max())
            assert np.allclose(r.traction.ravel(), trac, rtol=0, atol=1e-13 * np.abs(trac).max())
            # prescribed displacements come back as given, every frequency
            assert np.array_equal(r.disp.ravel()[d2.kode == 0], d2.bc[d2.kode == 0])
        outs[form] = (tmp_path / f"d_{form}").read_bytes()
    assert outs["plain"] == outs["mixed"]


def test_unknown_form_is_refused(tmp_path, golden_dir):
    with pytest.raises(ValueError):
        driver.run_case(os.path.join(golden_dir, "ESOLO240E_-5+5.DAT"),
                        os.path.join(golden_dir, "ESOLO240D_-5+5.DAT"),
                        tmp_path / "e", tmp_path / "d", form="fp16")


# src/analyser.py:12,27-34: how the reference's analysis script reads a run's log
_FLOAT = r"([-+]?(\d+(\.\d*)?|\.\d+)([eE][-+]?\d+)?)"
_ANALYSER = {"SHARED": r"Tempo gasto alocando os vetores compartilhados:\s*" + _FLOAT,
             "GHMATECE": r"GHMATECE: Tempo na ...:\s*" + _FLOAT,
             "GHMATECD": r"GHMATECD: Tempo na ...:\s*" + _FLOAT,
             "LINSOLVE": r"LINSOLVE: Tempo na ...:\s*" + _FLOAT,
             "INTEREC1": r"INTEREC1: Tempo na ...:\s*" + _FLOAT}


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_stage_log_reads_like_the_reference(tmp_path, golden_dir, form):
    ein = os.path.join(golden_dir, "ESOLO240E_-5+5.DAT")
    din = os.path.join(golden_dir, "ESOLO240D_-5+5.DAT")
    s = formats.read_static(ein)
    d = formats.read_dynamic(din, s.nbe)
    lines = []
    driver.run_case(ein, din, tmp_path / "e", tmp_path / "d", form=form,
                    solver_factory=_factory(d, []), log=lines.append)
    found = {}
    for ln in lines:
        for key, rx in _ANALYSER.items():
            m = re.search(rx, ln)
            if m:
                found[key] = float(m.group(1))
    want = {"SHARED", "GHMATECE", "INTEREC1"} | ({"GHMATECD", "LINSOLVE"} if form == "plain" else set())
    assert set(found) == want, lines
    assert all(v >= 0.0 for v in found.values())
    assert any(ln.strip().startswith("SWEEP: Tempo na GPU:") for ln in lines) == (form == "mixed")


def test_mixed_form_falls_back_to_fp64_where_refinement_stalls(tmp_path, golden_dir):
    ein = os.path.join(golden_dir, "ESOLO240E_-5+5.DAT")
    din = os.path.join(golden_dir, "ESOLO240D_-5+5.DAT")
    s = formats.read_static(ein)
    d = formats.read_dynamic(din, s.nbe)
    made, lines = [], []

    def make(st, device):
        sol = OracleSolver(st, d)
        sol.stall = (float(d.freqs[0]),)
        made.append(sol)
        return sol

    dout = tmp_path / "d"
    driver.run_case(ein, din, tmp_path / "e", dout, form="mixed", solver_factory=make, log=lines.append)
    assert made[0].fallbacks == [0]
    assert [c[2] for c in made[0].calls if c[0] == "sweep"] == ["mixed", "plain"]
    assert any("solved in FP64" in ln for ln in lines)
    with open(os.path.join(golden_dir, "SSOLO240D_-5+5.SOL"), "rb") as fh:
        assert dout.read_bytes() == fh.read()
