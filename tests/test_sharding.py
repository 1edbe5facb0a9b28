"""Multi-rank host logic of a sharded sweep, on CPU with the gloo backend (world size 2)."""
import os
import socket

import torch.multiprocessing as mp

from conftest import ROOT  # noqa: F401  (puts the repository on sys.path)
from cintx_b200.sharding import assign_chunks, chunks_of


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, costs, q):
    import sys
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from cintx_b200.sharding import assign_chunks, chunks_of, max_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    owner = assign_chunks(costs, world)
    mine = chunks_of(owner, rank)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    step_ms = 10.0 + rank  # each rank's own device time
    m = max_over_ranks(step_ms, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, gathered, m))


def test_assignment_covers_every_chunk_once():
    costs = [5.0, 1.0, 3.0, 3.0, 2.0, 8.0, 0.5]
    owner = assign_chunks(costs, 3)
    parts = [chunks_of(owner, r) for r in range(3)]
    assert sorted(c for p in parts for c in p) == list(range(len(costs)))
    loads = [sum(costs[c] for c in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)


def test_two_gloo_ranks_agree_and_reduce_max():
    costs = [float((7 * c) % 11 + 1) for c in range(23)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    g0, g1 = res[0][1], res[1][1]
    assert g0 == g1  # both ranks see the same assignment
    assert sorted(g0[0] + g0[1]) == list(range(len(costs))) and not set(g0[0]) & set(g0[1])
    assert res[0][2] == res[1][2] == 11.0  # max of the per-rank times


def test_chunk_size_per_world():
    from cintx_b200.sharding import chunk_doubles_for
    nint = 6_127_704_505  # mol120_spdf's sweep
    cap = 1 << 30
    assert chunk_doubles_for(nint, 1, cap) == cap
    for world in (2, 4, 8):
        cd = chunk_doubles_for(nint, world, cap)
        assert cd <= cap
        assert -(-nint // cd) >= 16 * world  # every rank gets about sixteen chunks to balance
    assert chunk_doubles_for(1000, 8, cap) == 1 << 22  # tiny sweeps keep a floor
