"""Replica logic of bench.py on CPU: max-over-ranks timing with two gloo ranks, the aggregate
per-step value, and the reference arm's silent exit on ranks other than 0."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        out[rank] = bench.max_over_ranks(10.0 + 5.0 * rank, world, "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        assert out[0] == out[1] == 15.0


def test_per_step_seconds_aggregates_replicas():
    sys.path.insert(0, ROOT)
    import bench
    # two replicas, three steps each, slowest rank 600 ms: six steps in 0.6 s
    assert bench.per_step_seconds(600.0, 3, 2) == pytest.approx(0.1)
    assert bench.per_step_seconds(600.0, 3, 1) == pytest.approx(0.2)


def test_reference_arm_other_ranks_exit_silently(capsys, monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    args = bench.argparse.Namespace(workload="incl129", sweeps=None)
    assert bench.run_reference_arm(args) == 0
    assert capsys.readouterr().out == ""
