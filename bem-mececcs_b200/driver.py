"""The reference's driver over its files: one mesh, every frequency.

`run_case` does what the reference's main program does with its four file
arguments (src/Main.for:85-200): read the static input and echo it
(INPUTECE), compute the static diagonals (GHMATECE), read the dynamic input
and echo it (INPUTECD), then per frequency assemble and solve (GHMATECD,
LINSOLVE), un-swap and evaluate the interior points (INTEREC) and append the
frequency's result block (OUTPUTEC).  The files it writes are the reference's
formats (formats.format_static_echo, formats.write_dynamic_output).

Frequencies are solved one at a time in FP64 (form "plain", what the
reference does), or all together by the lockstep sweep of the mixed form
(FP32 LU on tensor cores + FP64 refinement, form "mixed"), whose solutions
are un-swapped on the host; a frequency whose refinement does not converge
is solved again in FP64 (BemSolver.sweep's fallback).

Every frequency starts from the boundary conditions read from the file.  The
reference's CPU build un-swaps into its ZDFI array in place
(src/Interec.for:62-66 on the array set once at src/Main.for:158), so with
more than one frequency and any KODE = 0 its later frequencies start from the
previous frequency's tractions; that is not reproduced.  With one frequency
or KODE = 1 everywhere (the shipped cases) the two agree.  The reference also
lists FR, |ZFI(157)| and |ZFI(166)| on a unit it never opens
(src/Outputec.for:61, a compiler-named file); that side file is not written.
"""
from __future__ import annotations

import time

import numpy as np

from . import formats
from .solver import BemSolver, unswap_host

_ENC = "latin-1"
# A mixed-form problem whose last refinement step still changed the solution
# by more than this (relative) is solved again in FP64.
MIXED_FALLBACK_TOL = 1e-9


def run_case(input_e, input_d, output_e, output_d, *, form: str = "plain", refine: int = 3,
             device: int = 0, solver_factory=None, log=None) -> list:
    """Runs the case of the four files; returns the list of Results (one per
    frequency) that output_d holds.  `solver_factory(static, device)` makes
    the solver (BemSolver by default).  `log` (e.g. print), if given,
    receives the reference's stage-time lines ("Tempo gasto alocando os
    vetores compartilhados: <s>", "<ROUTINE>: Tempo na GPU: <s>" for
    GHMATECE and per frequency GHMATECD, LINSOLVE and INTEREC1; src/Main.for:
    135, src/Ghmatece.for:244-245, src/Ghmatecd.for:224-226,
    src/Linsolve.for:54-57, src/Interec.for:171-173), which the reference's
    analysis script reads.  The interior stresses are computed in the same
    kernel as the interior displacements, so INTEREC1 covers both and no
    SIGMAEC line is written; the mixed form's lockstep sweep reports one
    "SWEEP: Tempo na GPU: <s>" line in place of GHMATECD and LINSOLVE."""
    if form not in ("plain", "mixed"):
        raise ValueError(f"form must be 'plain' or 'mixed', not {form!r}")
    s = formats.read_static(input_e)
    with open(output_e, "w", encoding=_ENC) as fh:
        fh.write(formats.format_static_echo(s))
    make = solver_factory or (lambda st, dev: BemSolver(st, device=dev))
    t0 = time.perf_counter()
    sol = make(s, device)
    stage = _Stages(sol, log)
    stage.done("Tempo gasto alocando os vetores compartilhados:", t0)
    try:
        t0 = time.perf_counter()
        sol.ghmatece()
        stage.done("GHMATECE: Tempo na GPU:", t0)
        d = formats.read_dynamic(input_d, s.nbe)
        zdfi = np.asarray(d.bc, dtype=np.complex128)
        sol.set_bc(d.kode, zdfi, d.dam, d.rho)
        freqs = [float(f) for f in d.freqs]
        if form == "mixed" and freqs:
            t0 = time.perf_counter()
            x, _ = sol.sweep(freqs, form="mixed", batch=sol.sweep_batch_limit("mixed"), refine=refine,
                             fallback_tol=MIXED_FALLBACK_TOL)
            stage.done("SWEEP: Tempo na GPU:", t0)
            for i in sol.fallbacks:
                if log is not None:
                    log(f" MIXED: refinement did not converge at FR = {freqs[i]!r}; solved in FP64")
            bound = [unswap_host(x[i], d.kode, zdfi, sol.material[0]) for i in range(len(freqs))]
        else:
            bound = None
        results = []
        for i, fr in enumerate(freqs):
            if bound is not None:
                disp, trac = bound[i]
            else:
                t0 = time.perf_counter()
                sol.ghmatecd(fr)
                t0 = stage.done("GHMATECD: Tempo na GPU:", t0)
                sol.linsolve()
                stage.done("LINSOLVE: Tempo na GPU:", t0)
                disp, trac = sol.interec()
            if d.l > 0:
                t0 = time.perf_counter()
                zdsol, zssol = sol.interior(fr, disp, trac, d.cxi, d.cyi, d.czi)
                stage.done("INTEREC1: Tempo na GPU:", t0)
            else:
                zdsol, zssol = np.zeros(0, dtype=np.complex128), np.zeros(0, dtype=np.complex128)
            results.append(formats.Results(fr, np.asarray(disp).reshape(-1, 3),
                                           np.asarray(trac).reshape(-1, 3),
                                           np.asarray(zdsol).reshape(-1, 3),
                                           np.asarray(zssol).reshape(-1, 9)))
        formats.write_dynamic_output(output_d, s, d, sol.material, results)
        return results
    finally:
        sol.ctx.close()


class _Stages:
    """Stage timer: waits for the device, logs '<label> <seconds>' in the
    reference's list-directed style and returns the end time."""

    def __init__(self, sol, log):
        self.sol, self.log = sol, log

    def done(self, label: str, t0: float) -> float:
        if self.log is None:
            return time.perf_counter()
        self.sol.ctx.sync()
        t = time.perf_counter()
        self.log(f" {label} {t - t0:24.16E}")
        return t
