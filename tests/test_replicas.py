"""Replica mode (one rank per GPU, micrographs split in contiguous intervals) on CPU ranks
with the gloo backend: the host-side sharding and gathering, no GPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from replicas import run_replicas, work_intervals


def test_work_intervals_reference_rule():
    assert work_intervals(0, 10, 4) == [(0, 3), (3, 6), (6, 9), (9, 10)]
    assert work_intervals(0, 3, 8) == [(0, 1), (1, 2), (2, 3)]
    assert work_intervals(5, 6, 2) == [(5, 6)]
    assert work_intervals(0, 11, 2) == [(0, 6), (6, 11)]
    iv = work_intervals(0, 100, 8)
    assert iv[0][0] == 0 and iv[-1][1] == 100 and all(a[1] == b[0] for a, b in zip(iv, iv[1:]))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, first, last, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)

    def gather(obj):
        out = [None] * world
        dist.all_gather_object(out, obj)
        return out

    res = run_replicas(lambda i: (i, [i * 10 + k for k in range(i % 3)]), first, last, rank, world, gather)
    q.put((rank, res))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("first,last", [(0, 7), (2, 3)])
def test_replicas_two_ranks_gloo(first, last):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, first, last, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = [(i, [i * 10 + k for k in range(i % 3)]) for i in range(first, last)]
    assert results[0] == expect and results[1] == expect
