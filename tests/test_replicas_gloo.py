"""bench.py's N-GPU path (independent replicas, no data-path collective):
the rank aggregation and the reference arm's rank handling, run as two
gloo processes on the CPU (the GPU runs use the same code over NCCL)."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out):
    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws)
    try:
        # rank r ran for (r + 1) * 10 ms on 1000 * (r + 1) units
        ms, units, value = bench.replica_aggregate(10.0 * (rank + 1), 1000.0 * (rank + 1), ws)
        bench.barrier(ws)
        out[rank] = (ms, units, value)
    finally:
        dist.destroy_process_group()


def test_replica_aggregate_takes_max_time_and_total_units():
    ws = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(ws, _free_port(), out), nprocs=ws, start_method="spawn")
        res = dict(out)
    assert set(res) == {0, 1}
    for r in range(ws):
        ms, units, value = res[r]
        assert ms == 20.0 and units == 3000.0 and value == pytest.approx(3000.0 / 0.020)


def test_reference_arm_runs_on_rank_zero_only(capsys, monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")

    class Args:
        steps = 1
        warmup = 3

    bench.run_reference(Args())  # rank 1: no work, no output
    assert capsys.readouterr().out == ""
