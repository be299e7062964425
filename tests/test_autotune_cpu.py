"""The sweep autotuner's host logic on the CPU, against a fake solver.

The fake's sweep advances a fake clock by a cost that depends on the
context's switches and the lockstep batch, so the tuner's choice, the
switches it restores, the search space per form and the JSON cache can be
checked exactly, with no GPU.
"""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import __graft_entry__  # noqa: E402

__graft_entry__.load_package()
from bem_mececcs_b200 import autotune  # noqa: E402


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


class FakeCtx:
    def __init__(self, clock):
        self.clock = clock
        self.opts = {"lu_quads": True, "panel_calu": False, "lu_pairs": True, "tc_pair": True, "graphs": True}
        self.synced = 0

    def set_option(self, k, v):
        assert k in self.opts
        self.opts[k] = bool(v)

    def get_option(self, k):
        return self.opts[k]

    def sync(self):
        self.synced += 1


class FakeSolver:
    """Seconds per frequency: 1/10 with every switch at its default and the
    full batch of 7; each non-default switch and each missing batch slot makes
    it slower, except one planted better setting (graphs off)."""

    def __init__(self, nn=6480):
        self.clock = FakeClock()
        self.ctx = FakeCtx(self.clock)
        self.nn = nn
        self.calls = []

    def sweep_batch_limit(self, form):
        return 7 if form == "mixed" else 5

    def sweep(self, freqs, *, form, batch, refine, want_x):
        assert not want_x and len(freqs) % batch == 0
        o = self.ctx.opts
        per = 0.1
        per *= 1.0 if o["lu_quads"] else 1.3
        per *= 1.0 if o["lu_pairs"] else 1.2
        per *= 1.1 if o["panel_calu"] else 1.0
        per *= 1.0 if o["tc_pair"] else 1.1
        per *= 0.95 if not o["graphs"] else 1.0
        per *= 1.0 + 0.05 * (7 - batch)
        self.calls.append((form, batch, dict(o), len(freqs)))
        self.clock.t += per * len(freqs)


@pytest.fixture
def fake(monkeypatch):
    sol = FakeSolver()
    monkeypatch.setattr(autotune.time, "perf_counter", sol.clock)
    return sol


def test_picks_the_fastest_candidate_and_restores_the_switches(fake):
    before = dict(fake.ctx.opts)
    best = autotune.tune_sweep(fake, [1.0, 2.0, 3.0], form="mixed", steps=2)
    assert best["options"] == {"lu_quads": True, "panel_calu": False, "lu_pairs": True,
                               "tc_pair": True, "graphs": False}
    assert best["batch"] == 7
    assert best["solves_per_s"] == pytest.approx(1 / (0.1 * 0.95), rel=1e-3)
    # every combination of the default space x the batches {7, 6, 3}
    assert len(best["candidates"]) == 2 ** len(autotune.DEFAULT_SPACE) * 3
    assert {c["batch"] for c in best["candidates"]} == {7, 6, 3}
    assert fake.ctx.opts == before
    # too few frequencies are repeated to fill untimed + timed batches
    assert all(n in (b, b * 2) for (_, b, _, n) in fake.calls)


def test_fp64_form_tunes_only_graph_replay(fake):
    best = autotune.tune_sweep(fake, list(range(40)), form="plain", steps=1)
    assert set(best["options"]) == {"graphs"}
    assert {c["batch"] for c in best["candidates"]} == {5, 4, 2}
    assert all(f == "plain" for (f, _, _, _) in fake.calls)


def test_cache_roundtrip_applies_the_tuned_switches(fake, tmp_path):
    path = str(tmp_path / "sub" / "tune.json")
    best = autotune.tune_sweep(fake, list(range(30)), form="mixed", steps=1,
                               space={"graphs": (True, False), "lu_quads": (True, False)},
                               batches=[7, 4], cache_path=path)
    cache = json.load(open(path))
    key = autotune.cache_key(fake.nn, "mixed")
    assert list(cache) == [key] and cache[key]["batch"] == best["batch"]
    assert fake.ctx.opts["graphs"] is True  # restored after tuning
    cfg = autotune.tuned(fake, "mixed", path)
    assert cfg["options"] == {"graphs": False, "lu_quads": True}
    assert fake.ctx.opts["graphs"] is False  # applied
    # another size or form has no entry; a corrupt cache reads as empty
    assert autotune.tuned(FakeSolver(nn=999), "mixed", path) is None
    assert autotune.tuned(fake, "plain", path) is None
    open(path, "w").write("{not json")
    assert autotune.load_cache(path) == {}


def test_cache_keys_name_gpu_size_and_form():
    assert autotune.cache_key(6480, "mixed", gpu="NVIDIA B200") == "NVIDIA B200|nn=6480|form=mixed"
    assert autotune.cache_key(6480, "mixed", gpu="a") != autotune.cache_key(6480, "plain", gpu="a")
