"""Multi-GPU runs are independent replicas (one case per rank, no
collective on the data path); the bench reports the sum of all ranks'
particle-steps over the slowest rank's time. The reduction runs here on two
CPU ranks with the gloo backend."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.over_ranks(10.0 + 5.0 * rank, "max", "cpu")          # rank 1 is the slow one
        ps = bench.over_ranks(1.0e6 * (rank + 1), "sum", "cpu")
        q.put((rank, ms, ps))
    finally:
        dist.destroy_process_group()


def test_replica_aggregation_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, ps in got:
        assert ms == 15.0 and ps == 3.0e6


def test_single_process_is_its_own_aggregate():
    import bench
    assert bench.over_ranks(7.0, "max", "cpu") == 7.0
    assert bench.over_ranks(7.0, "sum", "cpu") == 7.0
