"""Precision at full size (the SC L=128 x 16-replica PT workload, bulk D=0.7, B=0.3, K=0.05):
over 1000 sweeps, every 100 sweeps, the device total energy (FP32 terms, FP64 sums) of every
replica's downloaded snapshot is compared with the FP64 oracle energy of the same spins, the
running FP64 accumulators (sums of per-sweep FP32 dE) with the recomputed energies, and the
winding number of all 128 z-slices (FP64 kernel) with the oracle, summed and rounded: two
replicas per block (rotating) and all 16 at the end."""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L, R, BLOCKS = 128, 16, 10


def _workers():
    try:
        return max(1, min(4, len(os.sched_getaffinity(0))))
    except Exception:
        return 1


def test_c3_energies_accumulators_and_winding_at_full_size(oracle, ib, cuda_ok):
    N = L ** 3
    op = oracle.Params(J=-1.0, Dz=0.7, B=0.3, K=0.05, dmi_bulk=True)
    pp = ib.params(J=-1.0, Dz=0.7, B=0.3, K=0.05, dmi="bulk")
    mesh = ib.ChainMesh.simple_cubic(L, n_replicas=R)
    mesh.init_uniform(0x15196)
    pt = ib.ParallelTempering(mesh, 1.0 / ib.temperature_ladder(0.1, 1.5, R), pp, seed=0x15196)
    nw = _workers()
    meshes = [oracle.Mesh.sc(L) for _ in range(nw)]   # one oracle mesh per worker thread

    def check(w, items):
        om = meshes[w]
        out = []
        for r, s, want_q in items:
            om.set_spins(s)
            e = om.canonical_energy(op)
            q = np.array([om.winding_number(z) for z in range(1, L + 1)]) if want_q else None
            out.append((r, e, q))
        return out

    worst_e = worst_acc = 0.0
    with ThreadPoolExecutor(nw) as ex:
        for block in range(BLOCKS):
            pt.run(10, 10)                                   # 100 sweeps, 10 exchanges
            e_run, _ = pt.energies()
            e_dev, _ = ib.observables(mesh, pp)
            # running accumulators vs recomputation: drift of 100-sweep blocks of FP32 dE sums
            worst_acc = max(worst_acc, float(np.max(np.abs(e_run - e_dev))) / N)
            assert np.max(np.abs(e_run - e_dev)) <= 1e-6 * N, (block, np.max(np.abs(e_run - e_dev)) / N)
            q_reps = set(range(R)) if block == BLOCKS - 1 else {(2 * block) % R, (2 * block + 1) % R}
            items = [(r, mesh.get_spins(r), r in q_reps) for r in range(R)]
            q_dev = {r: ib.winding_all_slices(mesh, r) for r in q_reps}
            parts = [items[w::nw] for w in range(nw)]
            for res in ex.map(check, range(nw), parts):
                for r, e_ref, q_ref in res:
                    worst_e = max(worst_e, abs(e_dev[r] - e_ref) / N)
                    assert abs(e_dev[r] - e_ref) <= 1e-6 * N, (block, r, e_dev[r], e_ref)
                    if q_ref is not None:
                        assert np.max(np.abs(q_dev[r] - q_ref)) < 1e-9, (block, r)
                        assert round(q_dev[r].sum()) == round(q_ref.sum()), (block, r)
    print(f"\nC3 precision over {BLOCKS * 100} sweeps: max |E_dev - E_fp64|/N {worst_e:.3e}, "
          f"max |E_acc - E_dev|/N {worst_acc:.3e}")
