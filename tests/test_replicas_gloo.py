"""The N-GPU bench path runs independent replicas ("replicas only"): the
process group is used only to time (max over ranks) and to sum the events.
This checks that reduction with two gloo ranks on the CPU."""
import os
import socket
import sys

import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seconds, events = bench.reduce_over_ranks(dist, seconds=1.5 + rank, events=100.0 * (rank + 1))
        out[rank] = (seconds, events)
    finally:
        dist.destroy_process_group()


def test_reduce_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    # every rank sees the slowest rank's time and the events of all replicas
    assert dict(out) == {0: (2.5, 300.0), 1: (2.5, 300.0)}


def test_reduce_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks(None, 2.0, 7.0) == (2.0, 7.0)
