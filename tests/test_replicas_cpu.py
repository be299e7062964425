"""The N > 1 path of bench.py on the CPU: two replicas as gloo ranks.

bench.py runs one independent replica per GPU: the 128-frequency sweep is
sharded by frequency, each rank solves its own share with no data exchange,
and the only collectives are the barrier before each timed region and one
MAX all-reduce of its time.  These tests drive the same helpers bench.py
uses (frequency_shard, max_over_ranks, job_rate, the reference arm's rank
filter) from world_size-2 gloo process groups on 127.0.0.1.
"""
import contextlib
import io
import json
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    from bem_mececcs_b200 import meshgen
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        r, w, _ = bench.dist_env()
        freqs = meshgen.sweep_frequencies(128, seed=3)
        mine = bench.frequency_shard(freqs, r, w)
        shares = [None] * w
        dist.all_gather_object(shares, [float(f) for f in mine])
        # three timed regions in bench.py's order (mixed, plain, e2e): a
        # barrier, then this rank's time, reduced to the slowest rank's
        times = {"mixed": 100.0 + 50.0 * r, "plain": 700.0 - 10.0 * r, "e2e": 101.0 + 60.0 * r}
        red = {}
        for k in ("mixed", "plain", "e2e"):
            dist.barrier()
            red[k] = bench.max_over_ranks(times[k], w, "cpu")
        # the reference arm: every rank but 0 leaves without work or output
        ref_out = None
        if r != 0:
            buf = io.StringIO()
            with contextlib.redirect_stdout(buf):
                ret = bench.run_reference(None)
            ref_out = {"ret": ret, "stdout": buf.getvalue()}
        with open(os.path.join(outdir, f"rank{r}.json"), "w") as fh:
            json.dump({"rank": r, "world": w, "mine": [float(f) for f in mine],
                       "shares": shares, "reduced": red,
                       "rate": bench.job_rate(w, 10 * 7, red["mixed"]), "ref": ref_out}, fh)
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def two_ranks(tmp_path_factory):
    import torch.multiprocessing as mp
    out = tmp_path_factory.mktemp("replicas")
    mp.start_processes(_rank_main, args=(2, _free_port(), str(out)), nprocs=2, join=True,
                       start_method="spawn")
    return [json.load(open(out / f"rank{r}.json")) for r in range(2)]


def test_shards_are_disjoint_and_cover_the_sweep(two_ranks):
    sys.path.insert(0, ROOT)
    from bem_mececcs_b200 import meshgen
    freqs = np.asarray(meshgen.sweep_frequencies(128, seed=3), dtype=np.float64)
    shares = two_ranks[0]["shares"]
    assert shares == two_ranks[1]["shares"]
    for r in range(2):
        assert two_ranks[r]["mine"] == shares[r]
    allf = np.concatenate([np.asarray(s) for s in shares])
    assert allf.size == freqs.size
    assert np.array_equal(np.sort(allf), np.sort(freqs))
    assert not set(shares[0]) & set(shares[1])
    assert abs(len(shares[0]) - len(shares[1])) <= 1


def test_times_reduce_to_the_slowest_rank_on_every_rank(two_ranks):
    for res in two_ranks:
        assert res["reduced"] == {"mixed": 150.0, "plain": 700.0, "e2e": 161.0}
        # value = units of all replicas over the slowest replica's time
        assert res["rate"] == pytest.approx(2 * 70 / 0.150)


def test_reference_arm_runs_on_rank_zero_only(two_ranks):
    ref = two_ranks[1]["ref"]
    assert ref == {"ret": None, "stdout": ""}


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shard_sizes_for_every_world(world):
    sys.path.insert(0, ROOT)
    import bench
    freqs = list(range(128))
    parts = [bench.frequency_shard(freqs, r, world) for r in range(world)]
    assert sorted(f for p in parts for f in p) == freqs
    assert max(map(len, parts)) - min(map(len, parts)) <= 1
    assert bench.max_over_ranks(12.5, 1, "cpu") == 12.5
