"""Host logic of the multi-GPU path: ensemble placement and the max-over-ranks timing
reduction, run as world_size-2 gloo process groups on the CPU."""
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


def _worker(rank, world, port, costs, q):
    import torch
    import torch.distributed as dist
    from ising_b200.sharding import partition_ensembles
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    mine = partition_ensembles(costs, world)[rank]
    # every rank derives the same placement; gather to check disjointness and coverage
    got = [None] * world
    dist.all_gather_object(got, mine)
    # timing reduction as bench.py does it: max over ranks
    t = torch.tensor([float(rank + 1) * 1.5], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    q.put((rank, got, float(t.item())))
    dist.destroy_process_group()


def test_two_rank_placement_and_timing():
    from ising_b200.sharding import ensemble_cost
    Ls = [16, 16, 24, 24, 32, 32, 48, 48, 64, 64, 96, 96]
    R = {16: 16, 24: 16, 32: 32, 48: 32, 64: 48, 96: 64}
    costs = [ensemble_cost(L, R[L], 10000) for L in Ls]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, tmax in res:
        assert tmax == 3.0
        flat = sorted(e for lst in got for e in lst)
        assert flat == list(range(len(Ls)))
        loads = [sum(costs[e] for e in lst) for lst in got]
        assert max(loads) / min(loads) < 1.05


def test_reference_slot_partition():
    from ising_b200.sharding import indices_from_slot, parameter_values, slot_from_indices, slot_partition
    NJ, ND, NB = 3, 4, 2
    n = NJ * ND * NB
    for size in (1, 2, 5):
        slots = [s for r in range(size) for s in slot_partition(n, r, size)]
        assert slots == list(range(1, n + 1))
    assert slot_partition(24, 4, 5) == list(range(17, 25))   # last rank takes the remainder
    for s in range(1, n + 1):
        assert slot_from_indices(NJ, ND, NB, *indices_from_slot(s, NJ, ND, NB)) == s
    assert parameter_values(1, NJ, ND, NB, -2.5, 2.5, -2.5, 2.5, 1.5, 1.5) == (-2.5, -2.5, 1.5)
    with pytest.raises(ValueError):
        slot_partition(3, 0, 4)
