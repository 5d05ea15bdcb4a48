"""Replicas across ranks (the path does not shard): bench.py's whole-job
value is all ranks' steps over the slowest rank's time.  Two gloo ranks on
CPU, rendezvous on 127.0.0.1."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        import bench
        secs = [2.0, 3.0][rank]
        q.put((rank, bench.max_over_ranks(secs, ws), bench.replica_value(10, secs, ws)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_value_takes_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, tmax, value in res:
        assert tmax == 3.0
        assert abs(value - 2 * 10 / 3.0) < 1e-12
