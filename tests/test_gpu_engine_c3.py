"""The persistent engine at the full C3 size (SC L=128 x 16 PT replicas, bulk D=0.7, B=0.3,
K=0.05, ball move r=0.2), on the schedules the autotuner chooses between: after 3 rounds of
10 sweeps its spins, exchange permutation and swap counts are bit-equal to the per-pass PT
path (itself replayed against the oracle) from the same seed; the spins stay unit vectors,
every z-slice's winding number is an integer, and the running FP64 accumulators agree with
energies recomputed from the spins within 1e-6 per site."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L, R, K_SWEEPS, ROUNDS, SEED = 128, 16, 10, 3, 0x15196


@pytest.mark.parametrize("sched", [dict(block_threads=128, chunk_pairs=8192, loader=0),
                                   dict(block_threads=256, chunk_pairs=16384, loader=1)],
                         ids=["registers", "staged"])
def test_engine_equals_pt_path_at_c3_size(ib, cuda_ok, sched):
    pp = ib.params(J=-1.0, Dz=0.7, B=0.3, K=0.05, dmi="bulk", include_Jp=False)
    betas = 1.0 / ib.temperature_ladder(0.1, 1.5, R)
    em = ib.ChainMesh.simple_cubic(L, n_replicas=R)
    rm = ib.ChainMesh.simple_cubic(L, n_replicas=R)
    em.init_uniform(SEED, 0)
    rm.init_uniform(SEED, 0)
    eng = ib.Ensembles([(em, betas, pp, 0)], seed=SEED)
    eng.set_schedule(**sched)
    eng.run(K_SWEEPS, ROUNDS)
    pt = ib.ParallelTempering(rm, betas, pp, seed=SEED, ensemble=0)
    pt.run(K_SWEEPS, ROUNDS)
    np.testing.assert_array_equal(eng.permutation(0), pt.permutation())
    a1, c1 = eng.swap_stats(0)
    a0, c0 = pt.swap_stats()
    np.testing.assert_array_equal(a1, a0)
    np.testing.assert_array_equal(c1, c0)
    N = em.numAtoms
    for r in range(R):
        s = em.get_spins(r)
        np.testing.assert_array_equal(s, rm.get_spins(r), err_msg=f"replica {r}")
        assert np.max(np.abs(np.linalg.norm(s, axis=1) - 1.0)) < 1e-6
    q = ib.winding_all_slices(em, int(eng.permutation(0)[0]))
    assert np.allclose(q, np.round(q), atol=1e-6)
    e_run, m_run = eng.energies(0)
    eng.resync()
    e_new, m_new = eng.energies(0)
    assert np.max(np.abs(e_run - e_new)) / N < 1e-6
    assert np.max(np.abs(m_run - m_new)) / N < 1e-6
    eng.close()
    pt.close()
