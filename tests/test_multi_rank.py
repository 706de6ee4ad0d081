"""The multi-GPU host path of bench.py on CPU: two gloo ranks (no GPU).

bench.py shards hypotheses over ranks (each rank tracks its own scenes), times
each rank on its device and reports the whole job's rate against the slowest
rank.  Here two processes run those pieces with the gloo backend: distinct
shards, the max-over-ranks reduction seen identically by both ranks, the
weak-scaling rate, and the reference arm doing no work on ranks other than 0.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
import bench  # noqa: E402
import scenes  # noqa: E402  (bench puts the package directory on sys.path)

WORLD = 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out_dir):
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=WORLD)
    try:
        # each rank's own shard of scenes
        tg, _ = scenes.generalized_3views_4pts(2, seed=bench.rank_seed(7, rank))
        shards = [None] * WORLD
        dist.all_gather_object(shards, tg)
        # the job's elapsed time is the slowest rank's
        local_ms = 100.0 + 50.0 * rank
        total_ms = bench.max_over_ranks(dist, local_ms, "cpu")
        rate = bench.whole_job_rate(WORLD, 2, 3, total_ms)
        dist.barrier()
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), total_ms=total_ms, rate=rate,
                 shard0=shards[0], shard1=shards[1])
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    mp.spawn(_rank_main, args=(_free_port(), str(tmp_path)), nprocs=WORLD, join=True)
    r = [np.load(os.path.join(tmp_path, "rank%d.npz" % k)) for k in range(WORLD)]
    for k in range(WORLD):
        assert float(r[k]["total_ms"]) == 150.0          # both ranks see the max
        assert float(r[k]["rate"]) == pytest.approx(WORLD * 2 * 3 / 0.150)
    assert not np.allclose(r[0]["shard0"], r[0]["shard1"])  # distinct hypotheses per rank
    assert np.array_equal(r[0]["shard1"], r[1]["shard1"])   # and every rank sees the same shards


def test_single_process_is_identity():
    assert bench.max_over_ranks(None, 12.5, "cpu") == 12.5
    assert bench.rank_seed(3, 0) != bench.rank_seed(3, 1)


def test_reference_arm_only_on_rank_zero():
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.reference_arm(None, 1) is None
    assert buf.getvalue() == ""
