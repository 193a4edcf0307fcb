"""CPU test of the multi-GPU path of bench.py: N independent replicas, one
process per rank, no collective on the data path — only the step-time max
and the work sum over ranks.  Two ranks on the gloo backend (127.0.0.1)."""
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
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took (10 + r) ms for 1000 * (r + 1) rays
        line = bench.replica_line(dist, rank, world, 10.0 + rank, 1000.0 * (rank + 1))
        bench.barrier(dist)
        out[rank] = line
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_max_time_and_total_work():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[1] is None
    line = out[0]
    assert line["n_gpus"] == 2 and line["ms_per_step"] == 11.0
    assert line["value"] == pytest.approx(3000.0 / 11e-3 / 1e6)


def test_single_process_has_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 3.5) == 3.5 and bench.sum_over_ranks(None, 2.0) == 2.0
    assert bench.replica_line(None, 0, 1, 4.0, 8e6) == {"ms_per_step": 4.0, "value": 2000.0, "n_gpus": 1}
