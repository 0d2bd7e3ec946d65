"""The persistent engine at the full C3 and C4 sizes.  C3 (SC L=128 x 16 PT replicas, bulk
D=0.7, B=0.3, K=0.05, ball move r=0.2), on the schedules the autotuner chooses between: after
3 rounds of 10 sweeps (every loader, the fused one with and without y-segments) its spins, exchange permutation and swap counts are bit-equal to the
per-pass PT path (itself replayed against the oracle) from the same seed; the spins stay unit
vectors, every z-slice's winding number is an integer, and the running FP64 accumulators
agree with energies recomputed from the spins within 1e-6 per site.  C4 (12 uneven
ensembles in one launch): after 2 rounds every ensemble's permutation, swap counts and first
and last replica equal those of its own per-pass PT run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L, R, K_SWEEPS, ROUNDS, SEED = 128, 16, 10, 3, 0x15196


@pytest.mark.parametrize("sched", [dict(block_threads=128, chunk_pairs=8192, loader=0),
                                   dict(block_threads=256, chunk_pairs=16384, loader=1),
                                   dict(block_threads=512, chunk_pairs=1 << 30, loader=2),
                                   dict(block_threads=256, chunk_pairs=16384, loader=2)],
                         ids=["registers", "staged", "fused", "fused-segments"])
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


@pytest.mark.parametrize("sched", [dict(block_threads=96, chunk_pairs=4096, loader=0),
                                   dict(block_threads=384, chunk_pairs=1 << 30, loader=2)],
                         ids=["registers-96", "fused-384"])
def test_engine_equals_pt_path_at_c5_shape(ib, cuda_ok, sched):
    """The default workload's mesh (SC L=96, nz = 96: rows of 24 lanes) on the schedules the
    autotuner picks for it, 12 of its 48 replicas, 2 rounds of 10 sweeps: bit-equal to the
    per-pass PT path."""
    L5, R5 = 96, 12
    pp = ib.params(J=-1.0, Dz=0.5, B=0.25, dmi="bulk", include_Jp=False)
    betas = 1.0 / ib.temperature_ladder(0.1, 1.5, R5)
    em = ib.ChainMesh.simple_cubic(L5, n_replicas=R5)
    rm = ib.ChainMesh.simple_cubic(L5, n_replicas=R5)
    em.init_uniform(SEED, 0)
    rm.init_uniform(SEED, 0)
    eng = ib.Ensembles([(em, betas, pp, 0)], seed=SEED, move=ib._lib.MOVE_BALL, r=0.2)
    eng.set_schedule(**sched)
    eng.run(K_SWEEPS, 2)
    pt = ib.ParallelTempering(rm, betas, pp, seed=SEED, ensemble=0, move=ib._lib.MOVE_BALL, r=0.2)
    pt.run(K_SWEEPS, 2)
    np.testing.assert_array_equal(eng.permutation(0), pt.permutation())
    for r in range(R5):
        np.testing.assert_array_equal(em.get_spins(r), rm.get_spins(r), err_msg=f"replica {r}")
    e_run, _ = eng.energies(0)
    eng.resync()
    e_new, _ = eng.energies(0)
    assert np.max(np.abs(e_run - e_new)) / em.numAtoms < 1e-6
    eng.close()
    pt.close()


# C4: 12 simple cubic ensembles, L in {16, 24, 32, 48, 64, 96} twice, 16-64 replicas each,
# (D, B) cycling over {0.3, 0.5, 0.7} x {0.1, 0.3}, T 0.1-2.0, bulk DMI, B along z (416
# replicas, 148,160,512 sites in one persistent launch)
C4_L = [16, 16, 24, 24, 32, 32, 48, 48, 64, 64, 96, 96]
C4_R = {16: 16, 24: 16, 32: 32, 48: 32, 64: 48, 96: 64}
C4_DB = [(0.3, 0.1), (0.3, 0.3), (0.5, 0.1), (0.5, 0.3), (0.7, 0.1), (0.7, 0.3)]


@pytest.mark.parametrize("sched", [dict(block_threads=128, chunk_pairs=32768, loader=0),
                                   dict(block_threads=384, chunk_pairs=1 << 30, loader=2)],
                         ids=["registers", "fused"])
def test_engine_equals_pt_path_at_c4_size(ib, cuda_ok, sched):
    spec, refs, emeshes, rmeshes = [], [], [], []
    for i, L in enumerate(C4_L):
        n = C4_R[L]
        D, B = C4_DB[i % 6]
        p = ib.params(J=-1.0, Dz=D, B=B, dmi="bulk", include_Jp=False)
        betas = 1.0 / ib.temperature_ladder(0.1, 2.0, n)
        em = ib.ChainMesh.simple_cubic(L, n_replicas=n)
        rm = ib.ChainMesh.simple_cubic(L, n_replicas=n)
        em.init_uniform(SEED, i)
        rm.init_uniform(SEED, i)
        emeshes.append(em)
        rmeshes.append(rm)
        spec.append((em, betas, p, i))
        refs.append((rm, betas, p, i))
    eng = ib.Ensembles(spec, seed=SEED)
    eng.set_schedule(**sched)
    eng.run(K_SWEEPS, 2)
    for i, (rm, betas, p, ens) in enumerate(refs):
        pt = ib.ParallelTempering(rm, betas, p, seed=SEED, ensemble=ens)
        pt.run(K_SWEEPS, 2)
        np.testing.assert_array_equal(eng.permutation(i), pt.permutation(), err_msg=f"ensemble {i}")
        a1, c1 = eng.swap_stats(i)
        a0, c0 = pt.swap_stats()
        np.testing.assert_array_equal(a1, a0)
        np.testing.assert_array_equal(c1, c0)
        n = len(betas)
        for r in (0, n - 1):
            np.testing.assert_array_equal(emeshes[i].get_spins(r), rm.get_spins(r),
                                          err_msg=f"ensemble {i} replica {r}")
        pt.close()
    eng.close()


@pytest.mark.parametrize("sched", [dict(block_threads=128, chunk_pairs=8192, loader=0),
                                   dict(block_threads=256, chunk_pairs=16384, loader=1),
                                   dict(block_threads=512, chunk_pairs=1 << 30, loader=2),
                                   dict(block_threads=256, chunk_pairs=16384, loader=2)],
                         ids=["registers", "staged", "fused", "fused-segments"])
def test_engine_long_run_at_c3_size(ib, cuda_ok, sched):
    """300 rounds (3000 sweeps) of the C3 workload in 3 launches: no wait gives up, the spins
    stay unit vectors, every slice charge stays an integer, and the running accumulators,
    summed from 3000 sweeps of FP32 dE, stay within 1e-6 per site of recomputed energies."""
    pp = ib.params(J=-1.0, Dz=0.7, B=0.3, K=0.05, dmi="bulk", include_Jp=False)
    betas = 1.0 / ib.temperature_ladder(0.1, 1.5, R)
    m = ib.ChainMesh.simple_cubic(L, n_replicas=R)
    m.init_uniform(SEED, 0)
    eng = ib.Ensembles([(m, betas, pp, 0)], seed=SEED)
    eng.set_schedule(**sched)
    for _ in range(3):
        eng.run(K_SWEEPS, 100)
    N = m.numAtoms
    for r in (0, R // 2, R - 1):
        s = m.get_spins(r)
        assert np.max(np.abs(np.linalg.norm(s, axis=1) - 1.0)) < 1e-6
        q = ib.winding_all_slices(m, r)
        assert np.allclose(q, np.round(q), atol=1e-6)
    perm = eng.permutation(0)
    assert sorted(perm) == list(range(R))
    e_run, m_run = eng.energies(0)
    eng.resync()
    e_new, m_new = eng.energies(0)
    assert np.max(np.abs(e_run - e_new)) / N < 1e-6
    assert np.max(np.abs(m_run - m_new)) / N < 1e-6
    att, acc = eng.swap_stats(0)
    assert np.all(att > 0) and np.all(acc <= att)
    eng.close()
