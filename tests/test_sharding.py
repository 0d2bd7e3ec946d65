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


# A small mix of uneven ensembles (L, temperatures, D, B, ensemble id), run with the oracle's
# FP64 colour-class sweeps and its restatement of the exchange: the chain of an ensemble is
# keyed by the seed and its global id, so a two-rank placement must give every ensemble the
# permutation and energies of the single-rank run.
MIX = [(4, 2, 0.3, 0.1, 11), (6, 3, 0.5, 0.3, 12), (8, 2, 0.7, 0.1, 13), (4, 4, 0.5, 0.2, 14), (6, 2, 0.3, 0.3, 15)]
MIX_SEED, MIX_K, MIX_ROUNDS = 0xC4, 2, 3


def _run_ensemble_cpu(O, L, n, D, B, ens):
    import numpy as np
    op = O.Params(J=-1.0, Dz=D, B=B, dmi_bulk=True)
    col = O.checkerboard(L, L, L)
    betas = 1.0 / O.temperature_ladder(0.1, 2.0, n)
    meshes = []
    for r in range(n):
        m = O.Mesh.sc(L)
        m.init_uniform(MIX_SEED, ens, r)
        meshes.append(m)
    t2r = list(range(n))
    for rnd in range(MIX_ROUNDS):
        for r, m in enumerate(meshes):
            key = O.SweepKey(seed=MIX_SEED, ensemble=ens, replica=r, move=1, r=0.2, philox_rounds=10)
            b = betas[t2r.index(r)]
            for sw in range(MIX_K):
                m.colour_pass(col, 0, rnd * MIX_K + sw, b, op, key)
                m.colour_pass(col, 1, rnd * MIX_K + sw, b, op, key)
        e_rep = np.array([m.canonical_energy(op) for m in meshes])
        _, perm = O.pt_exchange(MIX_SEED, ens, rnd, betas, e_rep, t2r)
        t2r = [int(v) for v in perm]
    return t2r, [float(v) for v in e_rep]


def _mix_worker(rank, world, port, q):
    import torch.distributed as dist
    from ising_b200.sharding import ensemble_cost, partition_ensembles
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    costs = [ensemble_cost(L, n, MIX_K * MIX_ROUNDS) for L, n, _, _, _ in MIX]
    mine = partition_ensembles(costs, world)[rank]
    res = {i: _run_ensemble_cpu(O, *MIX[i]) for i in mine}
    got = [None] * world
    dist.all_gather_object(got, res)
    dist.barrier()
    q.put((rank, mine, got))
    dist.destroy_process_group()


def test_two_rank_placement_reproduces_single_rank_chains(oracle):
    single = {i: _run_ensemble_cpu(oracle, *MIX[i]) for i in range(len(MIX))}
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_mix_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    owners = {}
    for rank, mine, got in res:
        assert mine, "every rank gets at least one ensemble of this mix"
        merged = {}
        for part in got:
            merged.update(part)
        assert sorted(merged) == list(range(len(MIX)))
        for i, (perm, en) in merged.items():
            assert perm == single[i][0], (i, perm, single[i][0])
            assert en == single[i][1], (i, en, single[i][1])
        for i in mine:
            assert i not in owners
            owners[i] = rank
    assert sorted(owners) == list(range(len(MIX)))


def test_members_for_rank_covers_every_ensemble_once():
    from ising_b200.sharding import members_for_rank

    class FakeMesh:
        def __init__(self, n):
            self.numAtoms = n

    members = [(FakeMesh(L ** 3), [1.0] * R, None, i) for i, (L, R) in
               enumerate([(16, 16), (16, 16), (24, 16), (32, 32), (64, 48), (96, 64)])]
    for world in (1, 2, 3, 8):
        seen = []
        for rank in range(world):
            idx, mine = members_for_rank(members, rank, world, sweeps=10)
            assert [m[3] for m in mine] == idx          # ensemble ids stay global
            seen += idx
        assert sorted(seen) == list(range(len(members)))
    with pytest.raises(ValueError):
        members_for_rank(members, 2, 2)
