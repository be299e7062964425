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


def _refine(a, b, steps):
    """The mixed form's refinement, restated in numpy: complex64 LU with
    partial pivoting (LAPACK cgetrf), then `steps` rounds of r = b - A x in
    FP64, d = LU32^-1 r, x += d.  Returns x and max|d|/max|x| of the last d."""
    from scipy.linalg import lu_factor, lu_solve
    lu = lu_factor(a.astype(np.complex64))
    x = lu_solve(lu, b.astype(np.complex64)).astype(np.complex128)
    corr = np.inf
    for _ in range(steps):
        r = b - a @ x
        d = lu_solve(lu, r.astype(np.complex64)).astype(np.complex128)
        x = x + d
        corr = np.abs(d).max() / np.abs(x).max()
    return x, corr


@pytest.mark.parametrize("cond", [1e1, 1e3, 1e5, 1e6, 1e7, 1e8, 1e9])
def test_fallback_threshold_separates_converged_from_stalled(cond):
    """Over conditioning from benign to beyond FP32: after 3 steps, a last
    correction <= 1e-9 (the driver's threshold) comes with an error <= 1e-8
    (the mixed form's target), and the systems FP32 factors cannot handle
    (cond * 2^-24 >= 1) all exceed the threshold and go to FP64."""
    rng = np.random.default_rng(int(np.log10(cond)))
    n = 160
    q1, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    q2, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    a = (q1 * np.logspace(0, -np.log10(cond), n)) @ q2.conj().T
    b = a @ (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    x_ref = np.linalg.solve(a, b)
    x, corr = _refine(a, b, 3)
    err = np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref)
    if corr <= 1e-9:
        assert err <= 1e-8, (cond, corr, err)
    if cond * 2.0 ** -24 >= 1.0:
        assert not corr <= 1e-9, (cond, corr, err)


class _FakeCtx:
    def __init__(self):
        self.closed = 0

    def close(self):
        self.closed += 1


def test_close_frees_only_a_context_the_solver_made():
    own = BemSolver.__new__(BemSolver)
    own._own_ctx, own.ctx = True, _FakeCtx()
    c = own.ctx
    with own as sol:
        assert sol is own
    assert c.closed == 1 and own.ctx is None
    own.close()  # twice is harmless
    assert c.closed == 1
    shared = BemSolver.__new__(BemSolver)
    shared._own_ctx, shared.ctx = False, _FakeCtx()
    shared.close()
    assert shared.ctx.closed == 0
