"""Placement of independent PT ensembles on ranks (one process per GPU).

Ensembles and (J, D, B) parameter slots never exchange data (src/PT.f90:147-176 farms them
over MPI ranks with only a barrier), so multi-GPU runs place whole ensembles on ranks and
need no collective on the data path.  Two placements:

- ``slot_partition`` restates the reference's contiguous slot blocks (PT.f90:147-166: each
  rank takes NumSlots / size slots, the last rank also the remainder) for drop-in drivers;
- ``partition_ensembles`` balances uneven ensembles by cost (sites x replicas x sweeps),
  longest-processing-time first.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def indices_from_slot(slot: int, NJ: int, ND: int, NB: int) -> Tuple[int, int, int]:
    """indicesFromSlot (src/PT-Utils.f90:11-22): 1-based slot -> 1-based (J, D, B) indices."""
    j = (slot - 1) // (ND * NB) + 1
    res = (slot - 1) % (ND * NB)
    return j, res // NB + 1, res % NB + 1


def slot_from_indices(NJ: int, ND: int, NB: int, j: int, d: int, b: int) -> int:
    """SlotFromIndices (src/PT-Utils.f90:24-30)."""
    return (j - 1) * ND * NB + (d - 1) * NB + b


def slot_partition(num_slots: int, rank: int, size: int) -> List[int]:
    """1-based slots of `rank` as src/PT.f90:147-166 assigns them."""
    if size < 1 or num_slots < size:
        raise ValueError("number of parameter slots must be at least the number of ranks")
    per = num_slots // size
    n = per + (num_slots % size if rank == size - 1 else 0)
    base = rank * per
    return [base + i for i in range(1, n + 1)]


def parameter_values(slot: int, NJ: int, ND: int, NB: int, Jmin, Jmax, Dmin, Dmax, Bmin, Bmax):
    """The (J, D, B) of a slot (src/PT.f90:171-175)."""
    j, d, b = indices_from_slot(slot, NJ, ND, NB)
    return ((j - 1) / NJ * (Jmax - Jmin) + Jmin, (d - 1) / ND * (Dmax - Dmin) + Dmin,
            (b - 1) / NB * (Bmax - Bmin) + Bmin)


def partition_ensembles(costs: Sequence[float], size: int) -> List[List[int]]:
    """Assign ensemble indices to `size` ranks, largest cost first onto the least loaded rank."""
    if size < 1:
        raise ValueError("size must be >= 1")
    load = [0.0] * size
    out: List[List[int]] = [[] for _ in range(size)]
    for e in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(size), key=lambda k: (load[k], k))
        out[r].append(e)
        load[r] += costs[e]
    for lst in out:
        lst.sort()
    return out


def ensemble_cost(L: int, replicas: int, sweeps: int, n_sub: int = 1) -> float:
    return float(L ** 3 * n_sub * replicas * sweeps)


def members_for_rank(members, rank: int, world: int, sweeps: int = 1):
    """(indices, members) that ``partition_ensembles`` places on `rank` of `world`.

    `members` is the engine's list of (mesh, betas, params, ensemble_id); the cost of an
    ensemble is its sites x temperatures x sweeps.  The ensemble ids stay those of the full
    list, so an ensemble's chain (keyed by seed and id) is the same on any placement."""
    if not 0 <= rank < world:
        raise ValueError("rank must be in 0..world-1")
    costs = [float(m.numAtoms) * len(b) * sweeps for m, b, _, _ in members]
    mine = partition_ensembles(costs, world)[rank]
    return mine, [members[i] for i in mine]

