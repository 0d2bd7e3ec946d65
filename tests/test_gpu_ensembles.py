"""Persistent multi-ensemble engine (ising_ensembles_*): every ensemble's spins, exchange
decisions and accumulators must equal those of the single-ensemble PT path
(ising_pt_*, itself replayed against the oracle in test_gpu_parity.py) run on its own mesh
with the same seed and ensemble id; the bounded waits must turn a flag that nothing sets
into ISING_ERR_TIMEOUT and leave the engine usable."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 0x15196

# (L, n_temps, D, B, K, ensemble id): uneven sizes and Hamiltonians, nz % 4 == 0
MEMBERS = [(8, 4, 0.3, 0.1, 0.0, 11), (12, 6, 0.5, 0.3, 0.0, 12), (16, 8, 0.7, 0.1, 0.0, 13), (8, 3, 0.5, 0.2, 0.0, 14)]


def _p(ib, D, B, K=0.0, dmi="bulk"):
    return ib.params(J=-1.0, Dz=D, B=B, K=K, dmi=dmi, include_Jp=False)


def _betas(ib, n):
    return 1.0 / ib.temperature_ladder(0.1, 2.0, n)


def _engine_and_refs(ib, members, k, rounds, scheme=0, move=1, sched=None, dmi="bulk"):
    """Runs the engine on fresh meshes and one ParallelTempering per member on twin meshes."""
    emeshes, rmeshes, spec = [], [], []
    for L, n, D, B, K, ens in members:
        nx, ny, nz = L if isinstance(L, tuple) else (L, L, L)
        em = ib.ChainMesh.simple_cubic(nx, ny=ny, nz=nz, n_replicas=n)
        rm = ib.ChainMesh.simple_cubic(nx, ny=ny, nz=nz, n_replicas=n)
        em.init_uniform(SEED, ens)
        rm.init_uniform(SEED, ens)
        emeshes.append(em)
        rmeshes.append(rm)
        spec.append((em, _betas(ib, n), _p(ib, D, B, K, dmi), ens))
    eng = ib.Ensembles(spec, seed=SEED, move=move, scheme=scheme)
    if sched:
        eng.set_schedule(**sched)
    eng.run(k, rounds)
    refs = []
    for (L, n, D, B, K, ens), rm in zip(members, rmeshes):
        pt = ib.ParallelTempering(rm, _betas(ib, n), _p(ib, D, B, K, dmi), seed=SEED, ensemble=ens, move=move,
                                  scheme=scheme)
        pt.run(k, rounds)
        refs.append(pt)
    return eng, emeshes, rmeshes, refs


def _assert_same(members, eng, emeshes, rmeshes, refs):
    for i, (L, n, *_rest) in enumerate(members):
        sites = int(np.prod(L)) if isinstance(L, tuple) else L ** 3
        for r in range(n):
            np.testing.assert_array_equal(emeshes[i].get_spins(r), rmeshes[i].get_spins(r),
                                          err_msg=f"ensemble {i} replica {r}")
        np.testing.assert_array_equal(eng.permutation(i), refs[i].permutation())
        e1, m1 = eng.energies(i)
        e0, m0 = refs[i].energies()
        # the running sums add FP32 per-block partials; block shapes differ between the two
        # paths, so they agree to FP32 rounding of the per-round increments
        np.testing.assert_allclose(e1, e0, rtol=1e-6, atol=1e-6 * n * sites)
        np.testing.assert_allclose(m1, m0, rtol=1e-6, atol=1e-6 * sites)
        a1, c1 = eng.swap_stats(i)
        a0, c0 = refs[i].swap_stats()
        np.testing.assert_array_equal(a1, a0)
        np.testing.assert_array_equal(c1, c0)


@pytest.mark.parametrize("sched", [
    None,
    {"block_threads": 128, "chunk_pairs": 16, "order": 0},          # one x-plane per task
    {"block_threads": 256, "chunk_pairs": 64, "order": 1, "group_bytes": 40_000},   # small replica groups
    {"block_threads": 64, "chunk_pairs": 100000, "order": 1, "group_bytes": 1},      # whole replicas, one per group
    {"block_threads": 128, "chunk_pairs": 16, "order": 2},          # wavefront order, one x-plane per task
    {"block_threads": 256, "chunk_pairs": 64, "order": 2},          # wavefront order, a few planes per task
])
def test_engine_matches_single_ensemble_pt(ib, cuda_ok, sched):
    eng, em, rm, refs = _engine_and_refs(ib, MEMBERS, k=3, rounds=5, sched=sched)
    _assert_same(MEMBERS, eng, em, rm, refs)


# nz = 128 meshes for the staged loader: plane groups that wrap in x (nx = 4: both halos),
# interior groups (nx = 12, 16), short y columns (ny = 4), uneven chunk tails (P = 8 of 12)
STAGED = [((12, 6, 128), 3, 0.5, 0.3, 0.05, 41), ((4, 4, 128), 2, 0.7, 0.1, 0.0, 42),
          ((16, 8, 128), 4, 0.3, 0.2, 0.0, 43)]


@pytest.mark.parametrize("chunk", [768, 1536, 2304, 100000])   # 4, 8, 12 planes, whole meshes
@pytest.mark.parametrize("move", [1, 0])
def test_staged_loader_matches_single_ensemble_pt(ib, cuda_ok, chunk, move):
    sched = {"block_threads": 256, "chunk_pairs": chunk, "order": 0, "loader": 1}
    eng, em, rm, refs = _engine_and_refs(ib, STAGED, k=3, rounds=4, move=move, sched=sched)
    assert eng.schedule()["loader"] == "staged"
    _assert_same(STAGED, eng, em, rm, refs)


def test_staged_loader_at_l128(ib, cuda_ok):
    members = [((128, 8, 128), 3, 0.7, 0.3, 0.05, 44)]
    sched = {"block_threads": 256, "chunk_pairs": 16384, "order": 0, "loader": 1}
    eng, em, rm, refs = _engine_and_refs(ib, members, k=2, rounds=3, sched=sched)
    _assert_same(members, eng, em, rm, refs)


def test_staged_loader_rejects_unsuited_meshes(ib, cuda_ok):
    spec = []
    for L, n, D, B, K, ens in MEMBERS[:2]:
        m = ib.ChainMesh.simple_cubic(L, n_replicas=n)
        m.init_uniform(SEED, ens)
        spec.append((m, _betas(ib, n), _p(ib, D, B), ens))
    eng = ib.Ensembles(spec, seed=SEED)
    with pytest.raises(ib.IsingError):
        eng.set_schedule(block_threads=256, chunk_pairs=4096, loader=1)      # nz != 128
    spec2 = []
    m = ib.ChainMesh.simple_cubic(12, ny=4, nz=128, n_replicas=2)
    m.init_uniform(SEED, 45)
    spec2.append((m, _betas(ib, 2), _p(ib, 0.5, 0.1), 45))
    eng2 = ib.Ensembles(spec2, seed=SEED)
    with pytest.raises(ib.IsingError):
        eng2.set_schedule(block_threads=128, chunk_pairs=4096, loader=1)     # blocks of 256 only
    eng2.set_schedule(block_threads=256, chunk_pairs=4096, loader=1)
    eng2.run(2, 1)


def test_staged_loader_timeout_and_recovery(ib, cuda_ok):
    spec = []
    for L, n, D, B, K, ens in STAGED[:2]:
        m = ib.ChainMesh.simple_cubic(L[0], ny=L[1], nz=L[2], n_replicas=n)
        m.init_uniform(SEED, ens)
        spec.append((m, _betas(ib, n), _p(ib, D, B), ens))
    eng = ib.Ensembles(spec, seed=SEED, wait_timeout_ms=50)
    eng.set_schedule(block_threads=256, chunk_pairs=768, loader=1)
    eng.inject_stall(1)
    with pytest.raises(ib.IsingError) as ei:
        eng.run(2, 3)
    assert ei.value.status == 4          # ISING_ERR_TIMEOUT
    eng.run(2, 2)
    for i in range(2):
        e_run, _ = eng.energies(i)
        assert np.all(np.isfinite(e_run))
        eng.resync()
        e_new, _ = eng.energies(i)
        assert np.max(np.abs(e_run - e_new)) / spec[i][0].numAtoms < 1e-5


def test_engine_random_pairs_and_uniform_move(ib, cuda_ok):
    members = MEMBERS[:3]
    eng, em, rm, refs = _engine_and_refs(ib, members, k=2, rounds=4, scheme=1, move=0)
    _assert_same(members, eng, em, rm, refs)


def test_engine_anisotropy_and_repeated_runs(ib, cuda_ok):
    members = [(8, 4, 0.3, 0.1, 0.05, 21), (12, 5, 0.7, 0.3, 0.05, 22)]
    eng, em, rm, refs = _engine_and_refs(ib, members, k=2, rounds=2)
    eng.run(2, 3)            # a second run continues the same chain
    for pt in refs:
        pt.run(2, 3)
    _assert_same(members, eng, em, rm, refs)


def test_engine_mixed_dmi_forms_stay_consistent(ib, cuda_ok):
    """Bulk and interfacial ensembles together use the tabulated-D kernel; the running FP64
    energies must agree with a full recomputation from the spins."""
    spec, meshes = [], []
    for i, (L, n, D, B, dmi) in enumerate([(8, 4, 0.5, 0.2, "bulk"), (12, 4, 0.5, 0.2, "interfacial")]):
        m = ib.ChainMesh.simple_cubic(L, n_replicas=n)
        m.init_uniform(SEED, 30 + i)
        meshes.append(m)
        spec.append((m, _betas(ib, n), _p(ib, D, B, 0.0, dmi), 30 + i))
    eng = ib.Ensembles(spec, seed=SEED)
    eng.run(3, 4)
    for i in range(2):
        e_run, m_run = eng.energies(i)
        eng.resync()
        e_new, m_new = eng.energies(i)
        n_sites = meshes[i].numAtoms
        assert np.max(np.abs(e_run - e_new)) / n_sites < 1e-5
        assert np.max(np.abs(m_run - m_new)) / n_sites < 1e-5


def test_bounded_wait_reports_timeout_and_engine_recovers(ib, cuda_ok):
    spec = []
    for L, n, D, B, K, ens in MEMBERS[:2]:
        m = ib.ChainMesh.simple_cubic(L, n_replicas=n)
        m.init_uniform(SEED, ens)
        spec.append((m, _betas(ib, n), _p(ib, D, B), ens))
    eng = ib.Ensembles(spec, seed=SEED, wait_timeout_ms=50)
    eng.inject_stall(1)
    with pytest.raises(ib.IsingError) as ei:
        eng.run(2, 3)
    assert ei.value.status == 4          # ISING_ERR_TIMEOUT
    eng.run(2, 2)            # usable again: no error, finite accumulators matching a resync
    for i in range(2):
        e_run, _ = eng.energies(i)
        assert np.all(np.isfinite(e_run))
        eng.resync()
        e_new, _ = eng.energies(i)
        assert np.max(np.abs(e_run - e_new)) / spec[i][0].numAtoms < 1e-5


def test_autotune_picks_a_timed_schedule(ib, cuda_ok):
    spec = []
    for L, n, D, B, K, ens in MEMBERS:
        m = ib.ChainMesh.simple_cubic(L, n_replicas=n)
        m.init_uniform(SEED, ens)
        spec.append((m, _betas(ib, n), _p(ib, D, B), ens))
    eng = ib.Ensembles(spec, seed=SEED)
    trials = eng.autotune(2, 1)
    assert len(trials) >= 10
    assert all(t["ms_per_round"] > 0 for t in trials)
    best = min(trials, key=lambda t: t["ms_per_round"])
    s = eng.schedule()
    assert (s["block_threads"], s["chunk_pairs"], s["order"]) == (best["block_threads"], best["chunk_pairs"], best["order"])
    eng.run(2, 2)


def test_engine_rejects_bad_input(ib, cuda_ok):
    m = ib.ChainMesh.simple_cubic(6, n_replicas=2)     # nz % 4 != 0: no colour-separated layout
    with pytest.raises(ib.IsingError):
        ib.Ensembles([(m, _betas(ib, 2), _p(ib, 0.3, 0.1), 1)])
    m8 = ib.ChainMesh.simple_cubic(8, n_replicas=2)
    with pytest.raises(ib.IsingError):
        ib.Ensembles([(m8, _betas(ib, 3), _p(ib, 0.3, 0.1), 1)])    # more temperatures than replicas
    with pytest.raises(ib.IsingError):
        ib.Ensembles([(m8, _betas(ib, 2), _p(ib, 0.3, 0.1), 1), (m8, _betas(ib, 2), _p(ib, 0.3, 0.1), 2)])
    eng = ib.Ensembles([(m8, _betas(ib, 2), _p(ib, 0.3, 0.1), 1)])
    with pytest.raises(ib.IsingError):
        eng.set_schedule(block_threads=48)
    with pytest.raises(ib.IsingError):
        eng.run(0, 1)


# The fused loader (both colour passes in one pass over ping-pong buffers) must reproduce the
# per-pass PT path bit for bit: chunks of 2 planes (many halo planes), chunks narrower than
# the mesh with uneven widths, whole meshes (halo planes are the chunk's own), y-segments of
# 2 rows and whole columns.
FUSED_SCHEDS = [
    {"block_threads": 128, "chunk_pairs": 16, "order": 0, "loader": 2},
    {"block_threads": 128, "chunk_pairs": 1 << 30, "order": 0, "loader": 2},
    {"block_threads": 256, "chunk_pairs": 64, "order": 0, "loader": 2},
    {"block_threads": 512, "chunk_pairs": 1 << 30, "order": 0, "loader": 2},
]


@pytest.mark.parametrize("sched", FUSED_SCHEDS)
@pytest.mark.parametrize("move", [1, 0])
def test_fused_loader_matches_single_ensemble_pt(ib, cuda_ok, sched, move):
    eng, em, rm, refs = _engine_and_refs(ib, MEMBERS, k=2, rounds=4, move=move, sched=sched)
    assert eng.schedule()["loader"] == "fused"
    _assert_same(MEMBERS, eng, em, rm, refs)


FUSED_WIDE = [((12, 6, 128), 3, 0.5, 0.3, 0.05, 51), ((4, 4, 128), 2, 0.7, 0.1, 0.0, 52),
              ((10, 8, 96), 4, 0.3, 0.2, 0.0, 53)]


@pytest.mark.parametrize("threads,chunk", [(128, 64), (256, 1 << 30), (384, 512), (512, 1 << 30)])
def test_fused_loader_nz128_and_nz96(ib, cuda_ok, threads, chunk):
    sched = {"block_threads": threads, "chunk_pairs": chunk, "order": 0, "loader": 2}
    eng, em, rm, refs = _engine_and_refs(ib, FUSED_WIDE, k=4, rounds=3, sched=sched)
    _assert_same(FUSED_WIDE, eng, em, rm, refs)


def test_fused_loader_random_pairs_anisotropy_and_repeated_runs(ib, cuda_ok):
    members = [(8, 4, 0.3, 0.1, 0.05, 61), (12, 5, 0.7, 0.3, 0.05, 62), (16, 3, 0.5, 0.2, 0.0, 63)]
    sched = {"block_threads": 256, "chunk_pairs": 32, "order": 0, "loader": 2}
    eng, em, rm, refs = _engine_and_refs(ib, members, k=2, rounds=2, scheme=1, sched=sched)
    eng.run(4, 2)            # a second run with another round length continues the same chain
    for pt in refs:
        pt.run(4, 2)
    _assert_same(members, eng, em, rm, refs)


def test_fused_loader_mixed_dmi_forms(ib, cuda_ok):
    """Bulk and interfacial ensembles together run the tabulated-D kernel."""
    members = [(8, 4, 0.5, 0.2, 0.0, 71), (12, 4, 0.5, 0.2, 0.0, 72)]
    emeshes, rmeshes, spec = [], [], []
    for (L, n, D, B, K, ens), dmi in zip(members, ("bulk", "interfacial")):
        em, rmm = ib.ChainMesh.simple_cubic(L, n_replicas=n), ib.ChainMesh.simple_cubic(L, n_replicas=n)
        em.init_uniform(SEED, ens)
        rmm.init_uniform(SEED, ens)
        emeshes.append(em)
        rmeshes.append(rmm)
        spec.append((em, _betas(ib, n), _p(ib, D, B, K, dmi), ens))
    eng = ib.Ensembles(spec, seed=SEED)
    eng.set_schedule(block_threads=128, chunk_pairs=16, loader=2)
    eng.run(2, 3)
    refs = []
    for (L, n, D, B, K, ens), dmi, rmm in zip(members, ("bulk", "interfacial"), rmeshes):
        pt = ib.ParallelTempering(rmm, _betas(ib, n), _p(ib, D, B, K, dmi), seed=SEED, ensemble=ens)
        pt.run(2, 3)
        refs.append(pt)
    _assert_same(members, eng, emeshes, rmeshes, refs)


def test_fused_loader_rejects_odd_rounds_and_small_blocks(ib, cuda_ok):
    m = ib.ChainMesh.simple_cubic(8, ny=8, nz=128, n_replicas=2)
    m.init_uniform(SEED, 81)
    eng = ib.Ensembles([(m, _betas(ib, 2), _p(ib, 0.3, 0.1), 81)], seed=SEED)
    with pytest.raises(ib.IsingError):
        eng.set_schedule(block_threads=96, chunk_pairs=4096, loader=2)     # fewer than nz threads
    eng.set_schedule(block_threads=128, chunk_pairs=4096, loader=2)
    with pytest.raises(ib.IsingError):
        eng.run(3, 1)                                                     # odd sweeps per round
    eng.run(2, 1)


def test_fused_loader_timeout_and_recovery(ib, cuda_ok):
    spec = []
    for L, n, D, B, K, ens in MEMBERS[:2]:
        m = ib.ChainMesh.simple_cubic(L, n_replicas=n)
        m.init_uniform(SEED, ens)
        spec.append((m, _betas(ib, n), _p(ib, D, B), ens))
    eng = ib.Ensembles(spec, seed=SEED, wait_timeout_ms=50)
    eng.set_schedule(block_threads=128, chunk_pairs=16, loader=2)
    eng.inject_stall(1)
    with pytest.raises(ib.IsingError) as ei:
        eng.run(2, 3)
    assert ei.value.status == 4          # ISING_ERR_TIMEOUT
    eng.run(2, 2)
    for i in range(2):
        e_run, _ = eng.energies(i)
        assert np.all(np.isfinite(e_run))
        eng.resync()
        e_new, _ = eng.energies(i)
        assert np.max(np.abs(e_run - e_new)) / spec[i][0].numAtoms < 1e-5


def test_set_resync_rearms_the_fp64_recomputation(ib, cuda_ok):
    spec = []
    for L, n, D, B, K, ens in MEMBERS[:2]:
        m = ib.ChainMesh.simple_cubic(L, n_replicas=n)
        m.init_uniform(SEED, ens)
        spec.append((m, _betas(ib, n), _p(ib, D, B), ens))
    eng = ib.Ensembles(spec, seed=SEED)
    eng.set_resync(3)
    eng.run(2, 6)               # ends on a resync: the accumulators equal a fresh recomputation
    e_run = [eng.energies(i)[0] for i in range(2)]
    eng.resync()
    for i in range(2):
        np.testing.assert_array_equal(e_run[i], eng.energies(i)[0])
    with pytest.raises(ib.IsingError):
        eng.set_resync(-1)
