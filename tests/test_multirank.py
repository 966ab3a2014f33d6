"""Multi-rank logic on CPU with gloo, world size 2 (no GPU)."""
import os
import socket

import pytest

from tictac_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dims = [24300, 24300, 42300, 42300, 53100, 53100, 56700, 56700]
        parts = shard.lpt_partition(shard.channel_weights(dims), world)
        mine = parts[rank]
        t = 1.0 + rank  # pretend step time
        tmax = shard.max_over_ranks(dist, t)
        got = shard.gather_to_rank0(dist, {c: complex(c, rank) for c in mine})
        if rank == 0:
            q.put((parts, tmax, got))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_gather():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    parts, tmax, got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert tmax == 2.0
    assert sorted(parts[0] + parts[1]) == list(range(8))
    # every channel solved exactly once, loads balanced within one channel's cost
    merged = {}
    for d in got:
        merged.update(d)
    assert sorted(merged) == list(range(8))
    w = shard.channel_weights([24300, 24300, 42300, 42300, 53100, 53100, 56700, 56700])
    loads = [sum(w[i] for i in p) for p in parts]
    assert abs(loads[0] - loads[1]) <= max(w)


def test_lpt_single_rank_and_energy_replicas():
    assert shard.lpt_partition([3.0, 1.0, 2.0], 1) == [[0, 1, 2]]
    assert shard.rank_lab_energies(10.0, 0) == 10.0 and shard.rank_lab_energies(10.0, 3) == 28.0
