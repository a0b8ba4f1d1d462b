"""The multi-GPU path of bench.py (independent replicas, max-over-ranks
timing) exercised with world_size 2 on the gloo backend, on CPU."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 100.0 + 50.0 * rank          # rank 1 is the slowest
        value, ms_max = bench.replica_throughput(1000, 10, ms, world)
        q.put((rank, value, ms_max, bench.max_over_ranks(float(rank), world)))
    finally:
        dist.destroy_process_group()


def test_replica_throughput_two_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, value, ms_max, mx in res:
        assert ms_max == 150.0
        assert abs(value - 2 * 1000 * 10 / 0.150) < 1e-6
        assert mx == 1.0
