"""Autotuner of the batched sweep (bem_sweep) for one GPU, mesh size and form.

The choices it makes are the library's algorithm switches and the lockstep
batch: the FP32 panel's pivoting (per column, or tournament per 8-column
sub-panel), four, two or one panels per tensor-core trailing update
(K = 256, 128 or 64; four take precedence where they fit), the update by CTA
pairs or by single CTAs, CUDA-graph replay
of the batch step, and the number of problems in lockstep (up to
bem_sweep_batch_limit).  Each candidate is timed on the
resident mesh on real frequencies (after one untimed batch) and the fastest
is kept in a JSON cache keyed by GPU, problem size and form, so that later
processes apply it without tuning again.

Every candidate computes the same solution to the refinement's accuracy; the
tuner only changes how fast.
"""
from __future__ import annotations

import itertools
import json
import os
import time

import numpy as np

DEFAULT_SPACE = {
    "lu_quads": (True, False),
    "panel_calu": (False, True),
    "lu_pairs": (True, False),
    "tc_pair": (True, False),
    "graphs": (True, False),
}


def _gpu_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown-gpu"


def cache_key(nn: int, form: str, gpu: str | None = None) -> str:
    return f"{gpu or _gpu_name()}|nn={nn}|form={form}"


def load_cache(path: str) -> dict:
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def save_cache(path: str, cache: dict) -> None:
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(cache, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def apply(sol, config: dict) -> None:
    """Sets the switches of a tuned configuration on the solver's context."""
    for k, v in config.get("options", {}).items():
        sol.ctx.set_option(k, v)


def _time_sweep(sol, freqs, form, batch, refine, steps) -> float:
    sol.sweep(freqs[:batch], form=form, batch=batch, refine=refine, want_x=False)  # untimed
    sol.ctx.sync()
    t0 = time.perf_counter()
    sol.sweep(freqs[: batch * steps], form=form, batch=batch, refine=refine, want_x=False)
    sol.ctx.sync()
    return batch * steps / (time.perf_counter() - t0)


def tune_sweep(sol, freqs, *, form: str = "mixed", refine: int = 3, steps: int = 2,
               space: dict | None = None, batches=None, cache_path: str | None = None) -> dict:
    """Times every candidate of `space` (option -> values) x `batches` on the
    solver's resident mesh; returns and (with cache_path) stores the best:
    {"options": {...}, "batch": B, "solves_per_s": V, "candidates": [...]}."""
    space = DEFAULT_SPACE if space is None else space
    if form != "mixed":  # the FP32 switches do not apply to the FP64 LU
        space = {k: v for k, v in space.items() if k == "graphs"}
    limit = sol.sweep_batch_limit(form)
    if batches is None:
        batches = sorted({limit, max(1, limit - 1), max(1, limit // 2)}, reverse=True)
    freqs = np.asarray(freqs, dtype=float)
    need = max(batches) * (steps + 1)
    if freqs.size < need:
        freqs = np.resize(freqs, need)
    keys = list(space)
    before = {k: sol.ctx.get_option(k) for k in keys}
    results = []
    for values in itertools.product(*(space[k] for k in keys)):
        opts = dict(zip(keys, values))
        for k, v in opts.items():
            sol.ctx.set_option(k, v)
        for b in batches:
            rate = _time_sweep(sol, freqs, form, b, refine, steps)
            results.append({"options": opts, "batch": b, "solves_per_s": round(rate, 3)})
    for k, v in before.items():
        sol.ctx.set_option(k, v)
    best = max(results, key=lambda r: r["solves_per_s"])
    out = dict(best)
    out["candidates"] = results
    if cache_path:
        cache = load_cache(cache_path)
        cache[cache_key(sol.nn, form)] = out
        save_cache(cache_path, cache)
    return out


def tuned(sol, form: str, cache_path: str) -> dict | None:
    """The cached configuration for this GPU, size and form, applied to the
    solver's context; None when there is none."""
    cfg = load_cache(cache_path).get(cache_key(sol.nn, form))
    if cfg:
        apply(sol, cfg)
    return cfg
