"""The multi-process plumbing of bench.py on CPU: world_size 2 over gloo
(127.0.0.1).  bench.py runs one replica per GPU (the step has no cross-rank
exchange), so its distributed parts are the max-over-ranks timing, the
rank-0-only output and the reference arm's rank-0-only run."""
import contextlib
import io
import os
import socket
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        assert bench._dist() == (ws, rank, rank)
        # every rank's own time, the job's time is the slowest rank's
        t = bench._max_over_ranks(10.0 + rank, ws, torch.device("cpu"))
        # the reference arm: ranks other than 0 exit 0 without work or output
        buf = io.StringIO()
        if rank != 0:
            with contextlib.redirect_stdout(buf):
                rc = bench.main(["--impl", "reference", "--gpus", str(ws), "--steps", "1", "--warmup", "0",
                                 "--workload", "tgv32"])
        else:
            rc = 0
        dist.barrier()
        out.put((rank, t, rc, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_and_rank0_output():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [11.0, 11.0]
    assert res[1][2] == 0 and res[1][3] == ""


def test_replica_throughput_aggregates_over_ranks():
    sys.path.insert(0, str(ROOT))
    import bench
    # weak scaling: N replicas each process `cells` cells per stage
    v1 = bench._throughput(cells=1000, steps=10, ms=20.0, ws=1)
    v4 = bench._throughput(cells=1000, steps=10, ms=20.0, ws=4)
    assert v4 == pytest.approx(4 * v1)
    assert v1 == pytest.approx(1000 * 3 * 10 / 0.02 / 1e6)
