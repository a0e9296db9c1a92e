"""bench.py's multi-rank plumbing (replicas, one per GPU): timing is the
maximum over ranks and the value aggregates every rank's replica.  Two gloo
ranks on the CPU exercise the same collective the NCCL run uses."""

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(10.0 + 5.0 * rank, world)
        q.put((rank, t, bench.replica_value(1000, world, 4, t)))
    finally:
        dist.destroy_process_group()


def test_timing_is_the_slowest_rank_and_value_aggregates_replicas():
    import bench

    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_value(1000, 1, 4, 2000.0) == 2000.0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [15.0, 15.0]  # both ranks report the slower rank's time
    assert got[0][2] == pytest.approx(2 * 1000 * 4 / 0.015)


def test_hbm_peak_reads_the_measured_file_or_falls_back():
    import bench

    v, basis = bench.hbm_peak()
    assert v > 1000 and basis in ("measured", "fallback")
    if (ROOT / "MEASURED_PEAKS.json").exists():
        assert basis == "measured"
