"""The multi-GPU path of bench.py on CPU: two gloo ranks stand in for two
replicas.  Each rank renders its own seeds (no collective on the data path);
the job's time is the slowest rank's and its samples are all ranks' samples."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        # rank r "took" 100 + 50 r ms for 1000 (r + 1) samples
        value, ms_max, samples = bench.job_throughput(100.0 + 50.0 * rank, 1000 * (rank + 1), torch.device("cpu"), world)
        seeds = [bench.replica_seed(rank, k) for k in range(5)]
        q.put((rank, value, ms_max, samples, seeds))
    finally:
        dist.destroy_process_group()


def test_two_replicas_on_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, ms_max, samples, seeds in res:
        assert ms_max == pytest.approx(150.0)          # the slowest rank's time
        assert samples == 3000                           # all ranks' samples
        assert value == pytest.approx(3000 / 0.150 / 1e6)
    # replicas never render the same samples
    assert not set(res[0][4]) & set(res[1][4])


def test_single_process_needs_no_group():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    value, ms_max, samples = bench.job_throughput(200.0, 4000, torch.device("cpu"), 1)
    assert (ms_max, samples) == (200.0, 4000) and value == pytest.approx(4000 / 0.2 / 1e6)
