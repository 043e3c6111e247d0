"""Two ranks on the CPU (gloo): the data path shards without any exchange, and the bench's
reductions (max of per-rank times, sum of work) agree with the single-process numbers."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from directsht_b200.dist import reduce_scalar, shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from directsht_b200.serve import Admission
        ids = shard(list(range(23)), rank, world)
        # each rank admits its own requests under its own budget (no cross-rank traffic)
        a = Admission(budget_bytes=10**9, slots=4)
        for i in ids:
            a.push(i, 1000 + i)
        done = []
        while a.queue:
            start, _ = a.pop_admissible()
            for r, fp in start:
                done.append(r)
                a.release(fp)
        t_rank = 1.0 + rank  # per-rank device time
        out[rank] = (sorted(done), reduce_scalar(t_rank, "max"), reduce_scalar(len(done), "sum"))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_ranks_shard_and_reduce():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    assert sorted(res[0][0] + res[1][0]) == list(range(23))
    assert not set(res[0][0]) & set(res[1][0])
    for r in range(world):
        assert res[r][1] == 2.0 and res[r][2] == 23
