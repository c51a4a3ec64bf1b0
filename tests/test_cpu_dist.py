"""The multi-process plumbing of bench.py (one process per GPU, replicas
only): barrier and max-over-ranks timing, run here as two gloo ranks on the
CPU."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    bench.barrier(world)
    got = bench.max_over_ranks(10.0 + rank, world)
    bench.barrier(world)
    dist.destroy_process_group()
    q.put((rank, got))


def test_two_rank_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 11.0, 1: 11.0}


def test_degenerate_element_raises_before_any_gpu_work():
    import numpy as np

    import redbirdpy_b200 as rbb
    from redbirdpy_b200.meshgen import kuhn_box

    node, elem = kuhn_box([2, 2, 2], 1)
    node = node.copy()
    elem = elem.copy()
    elem[0, 3] = elem[0, 2]  # a repeated node: zero volume
    cfg = dict(node=node, elem=elem, prop=np.array([[0, 0, 1, 1], [0.01, 1.0, 0, 1.37]]),
               srcpos=np.array([[1, 1, 0.0]]), srcdir=np.array([[0, 0, 1.0]]), detpos=np.array([[1.5, 1, 0.0]]))
    with pytest.raises(ValueError, match="Degenerate"):
        rbb.meshprep(cfg)
