"""Precision at full size (the SC L=128 x 16-replica PT workload, bulk D=0.7, B=0.3, K=0.05):
every 100 sweeps the device total energy (FP32 terms, FP64 sums) of downloaded snapshots is
compared with the FP64 oracle energy of the same spins, the running FP64 accumulators (sums of
per-sweep FP32 dE) with the recomputed energies, and the winding number of every one of the
128 z-slices (FP64 kernel) with the oracle, summed and rounded."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_c3_energies_accumulators_and_winding_at_full_size(oracle, ib, cuda_ok):
    L, R = 128, 16
    N = L ** 3
    op = oracle.Params(J=-1.0, Dz=0.7, B=0.3, K=0.05, dmi_bulk=True)
    pp = ib.params(J=-1.0, Dz=0.7, B=0.3, K=0.05, dmi="bulk")
    mesh = ib.ChainMesh.simple_cubic(L, n_replicas=R)
    mesh.init_uniform(0x15196)
    pt = ib.ParallelTempering(mesh, 1.0 / ib.temperature_ladder(0.1, 1.5, R), pp, seed=0x15196)
    om = oracle.Mesh.sc(L)
    for block in range(3):
        pt.run(10, 10)                                   # 100 sweeps, 10 exchanges
        e_run, _ = pt.energies()
        e_dev, _ = ib.observables(mesh, pp)
        # running accumulators vs recomputation: drift of 100-sweep blocks of FP32 dE sums
        assert np.max(np.abs(e_run - e_dev)) <= 1e-6 * N, np.max(np.abs(e_run - e_dev)) / N
        for r in (0, 7, 15):
            s = mesh.get_spins(r)
            om.set_spins(s)
            e_ref = om.canonical_energy(op)
            assert abs(e_dev[r] - e_ref) <= 1e-6 * N, (r, e_dev[r], e_ref)
            q_dev = ib.winding_all_slices(mesh, r)
            q_ref = np.array([om.winding_number(z) for z in range(1, L + 1)])
            assert np.max(np.abs(q_dev - q_ref)) < 1e-9
            assert round(q_dev.sum()) == round(q_ref.sum())
