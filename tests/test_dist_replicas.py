"""The multi-GPU path of bench.py is replicas only: every rank advances its
own copy of the case, ranks meet at a barrier, and the timing is the maximum
over ranks. Exercised here with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q, vis):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    if vis is None:
        os.environ.pop("CUDA_VISIBLE_DEVICES", None)
    else:
        os.environ["CUDA_VISIBLE_DEVICES"] = vis
    import bench

    d = bench.Dist(world)
    d.barrier()
    mx = d.max(1.0 + rank)           # rank r "took" 1 + r ms
    q.put((rank, mx, os.environ.get("CUDA_VISIBLE_DEVICES")))
    d.close()


@pytest.mark.timeout(120)
@pytest.mark.parametrize("vis,expect", [(None, ["0", "1"]), ("4,5", ["4", "5"])])
def test_two_gloo_ranks_take_the_max(vis, expect):
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q, vis)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    assert [g[1] for g in got] == [2.0, 2.0]
    # one process per GPU: each rank sees only its own device
    assert [g[2] for g in got] == expect
