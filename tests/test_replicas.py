"""CPU, two gloo ranks: the replica timing of bench.py --gpus N (one process
per GPU, independent batches) combines the ranks' device times by their
maximum and their units by their sum."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    from libdescriptor_b200.replicas import replica_throughput

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        units = 1000.0 * (rank + 1)          # uneven work per rank
        ms = 10.0 + 5.0 * rank               # rank 1 is the slowest
        rate, ms_max, total = replica_throughput(units, ms, dist, torch.device("cpu"))
        q.put((rank, rate, ms_max, total))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_replica_throughput_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rate, ms_max, total in out:
        assert ms_max == 15.0
        assert total == 3000.0
        assert abs(rate - 3000.0 / 0.015) < 1e-6


def test_replica_throughput_single_process():
    from libdescriptor_b200.replicas import replica_throughput

    rate, ms, total = replica_throughput(500.0, 2.0)
    assert (rate, ms, total) == (250000.0, 2.0, 500.0)
