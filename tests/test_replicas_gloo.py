"""Replica bookkeeping over two ranks (gloo, CPU): shards, gather, max over ranks.
The per-rank transform is the oracle standing in for the GPU plans."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cuhpx_b200 import replicas
from oracle import hpx_oracle as O


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nside, L = 4, 7
        rng = np.random.default_rng(0)
        f = torch.from_numpy(rng.standard_normal((5, 12 * nside * nside)))  # same batch on every rank
        mine = replicas.local_shard(f)
        a = torch.from_numpy(O.sht(mine.numpy(), nside, L, L)) if mine.shape[0] else torch.zeros((0, L, L),
                                                                                                 dtype=torch.complex128)
        full = replicas.gather_shards(torch.view_as_real(a).contiguous(), f.shape[0])
        t = replicas.max_over_ranks(10.0 * (rank + 1))
        if rank == 0:
            ref = O.sht(f.numpy(), nside, L, L)
            out.put((float(np.abs(torch.view_as_complex(full).numpy() - ref).max()), t, tuple(mine.shape)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_shard_range_partitions():
    for n in (0, 1, 5, 64, 97):
        for world in (1, 2, 3, 8):
            spans = [replicas.shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[r][1] == spans[r + 1][0] for r in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    err, tmax, shape = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert err < 1e-12
    assert tmax == 20.0
    assert shape == (3, 192)
