"""BemSolver.sweep's FP64 fallback for mixed-form problems whose refinement
does not converge, on the CPU: the raw sweep is replaced by a fake that
returns chosen corrections, so the selection and the re-solve are checked
exactly."""
import numpy as np
import pytest

from bem_mececcs_b200.solver import BemSolver


class FakeRaw(BemSolver):
    def __init__(self, corr):
        self.nn = 3
        self.corr = np.asarray(corr, dtype=float)
        self.raw_calls = []

    def _sweep_raw(self, freqs, form, batch, refine, want_x):
        freqs = np.asarray(freqs, dtype=float)
        self.raw_calls.append((form, batch, refine, freqs.tolist()))
        tag = 1.0 if form == "mixed" else 2.0  # which form produced a row
        x = np.outer(freqs, np.ones(self.nn)) * tag + 0j
        corr = self.corr.copy() if form == "mixed" else np.zeros(freqs.size)
        return x, corr

    def sweep_batch_limit(self, form="mixed"):
        return 7 if form == "mixed" else 4


def test_stalled_and_non_finite_problems_are_solved_in_fp64():
    sol = FakeRaw([1e-15, 3e-6, np.nan, 1e-12, np.inf])
    freqs = [0.5, 1.0, 2.0, 4.0, 8.0]
    x, corr = sol.sweep(freqs, form="mixed", batch=7, refine=3, fallback_tol=1e-9)
    assert sol.fallbacks == [1, 2, 4]
    assert sol.raw_calls[1] == ("plain", 4, 3, [1.0, 2.0, 8.0])
    for i, f in enumerate(freqs):
        assert np.all(x[i] == f * (2.0 if i in (1, 2, 4) else 1.0))
    assert corr[1] == 3e-6 and np.isnan(corr[2])  # reported as measured


@pytest.mark.parametrize("kw", [dict(fallback_tol=None), dict(fallback_tol=1e-9, refine=0),
                                dict(fallback_tol=1e-9, form="plain"),
                                dict(fallback_tol=1e-9, want_x=False)])
def test_no_fallback_unless_asked_for_mixed_refined_solutions(kw):
    args = dict(form="mixed", batch=7, refine=3, want_x=True)
    args.update(kw)
    sol = FakeRaw([1e-3, 1e-3])
    sol.sweep([1.0, 2.0], **args)
    assert sol.fallbacks == [] and len(sol.raw_calls) == 1


def test_converged_problems_are_left_alone():
    sol = FakeRaw([1e-15, 2e-14])
    x, _ = sol.sweep([1.0, 2.0], form="mixed", batch=2, refine=3, fallback_tol=1e-9)
    assert sol.fallbacks == [] and len(sol.raw_calls) == 1 and np.all(x.real[:, 0] == [1.0, 2.0])
