"""The multi-GPU form of the path is replicas: each rank parses its own
document with no collective on the data path; the bench takes the slowest
rank's device time and reports whole-job throughput. These tests run that
host logic on two gloo ranks on the CPU."""

import os
import socket

import pytest
import torch.multiprocessing as mp

import bench
from alpacc_b200 import workloads as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        q.put((rank, bench.max_over_ranks(dist, ms)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got == {0: 15.0, 1: 15.0}


def test_single_process_needs_no_group():
    assert bench.max_over_ranks(None, 7.5) == 7.5


def test_job_throughput_counts_every_rank():
    n = 256 << 20
    one = bench.job_throughput(1, n, 10, 100.0)
    assert one == pytest.approx(n * 10 / 0.1 / 1e9)
    assert bench.job_throughput(4, n, 10, 100.0) == pytest.approx(4 * one)


def test_ranks_parse_different_documents():
    # each rank's document is seeded by its rank (weak scaling, no shared input)
    assert W.json_doc(1 << 16, 2) != W.json_doc(1 << 16, 3)


def test_reference_arm_prints_only_on_rank_zero(capsys):
    class A:
        size = 1 << 20
        gpus = 2
        steps = 1
        warmup = 0
        ref_sample = 1 << 20
        workload = "json"

    bench.reference_arm(A, 1, 2)
    assert capsys.readouterr().out == ""
