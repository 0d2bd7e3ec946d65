"""The storage orders and colour classes of the reference's own lattices (src/PT.f90:145,
src/ISING.f90:105) against the FP64 oracle: BCC in sublattice planes (layout 3; without J'
the two sublattices are the classes and run on the sublattice-class kernel, with J' a greedy
colouring runs on the stencil kernel), hyper-kagome with even extents in octant order.  Spins
round-trip through the layout, per-site and total energies and winding numbers equal the
oracle's, and sweeps replay the oracle's colour passes (same Philox keys, the product's colour
classes) decision for decision, with J' on (BCC's shell 2 holds each site itself, which the
classes accept) and off, both moves, over several sweeps."""
import numpy as np
import pytest

from test_gpu_parity import _both_params, _pair, _random_spins

pytestmark = pytest.mark.gpu

LAYOUT = {"BCC": "sublattice", "HK": "octant"}
CASES = [
    ("BCC", (6, 6, 4), dict(J=-1.0, Dz=0.4, B=0.1, bulk=True), 1, 0.2, 1.5),
    ("BCC", (5, 6, 8), dict(J=-1.0, Dz=0.5, B=0.2, bulk=False), 1, 0.3, 1.2),
    ("BCC", (4, 4, 6), dict(J=1.0, Dz=0.3, B=-0.2, K=0.1, bulk=False), 0, 0.0, 2.5),
    ("BCC", (4, 6, 8), dict(J=-1.0, Jp=0.2, Dz=0.3, B=0.2, K=0.05, bulk=False), 0, 0.0, 2.0),
    ("HK", (4, 4, 4), dict(J=-1.0, Dz=0.3, B=0.1, bulk=False), 1, 0.25, 1.0),
    ("HK", (4, 6, 4), dict(J=1.0, Jp=0.1, Dz=0.2, B=0.3, bulk=True), 0, 0.0, 3.0),
    # 15 block classes with J' on the pair kernel (nz % 4 == 0) and on the one-site kernel
    ("HK", (8, 8, 8), dict(J=-1.0, Jp=0.1, Dz=0.3, B=0.1, bulk=False), 1, 0.2, 1.5),
    ("HK", (4, 4, 6), dict(J=-1.0, Jp=-0.2, Dz=0.4, B=0.2, bulk=False), 1, 0.3, 2.0),
    ("HK", (6, 4, 6), dict(J=-1.0, Dz=0.4, B=0.2, bulk=False), 0, 0.0, 1.2),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_octant_layout_energies_and_winding(oracle, ib, cuda_ok, case):
    kind, dims, h, _, _, _ = CASES[case]
    om, pm = _pair(oracle, ib, kind, dims, n_replicas=2)
    assert pm.layout == LAYOUT[kind]
    s = _random_spins(om.natoms, 300 + case)
    om.set_spins(s)
    pm.set_spins(s, 1)
    np.testing.assert_array_equal(pm.get_spins(1), s)
    op, pp = _both_params(oracle, ib, **h)
    rng = np.random.default_rng(case)
    atoms = rng.choice(om.natoms, size=min(300, om.natoms), replace=False)
    sp = _random_spins(len(atoms), 900 + case)
    go, gn = ib.local_energy_batch(pm, atoms, sp, pp, replica=1)
    for k, a in enumerate(atoms):
        o, n = om.local_energy(int(a), op, sp[k])
        scale = 1.0 + abs(o)
        assert abs(go[k] - o) < 1e-6 * scale * 10 and abs(gn[k] - n) < 1e-6 * scale * 10, (a, go[k], o)
    e, _ = ib.observables(pm, pp)
    assert abs(e[1] - om.canonical_energy(op)) < 1e-6 * om.natoms
    q = ib.winding_all_slices(pm, 1)
    for z in range(1, dims[2] + 1):
        assert abs(q[z - 1] - om.winding_number(z)) < 1e-9


@pytest.mark.parametrize("case", range(len(CASES)))
def test_octant_sweeps_replay_the_oracle(oracle, ib, cuda_ok, case):
    kind, dims, h, move, r, beta = CASES[case]
    om, pm = _pair(oracle, ib, kind, dims)
    s = _random_spins(om.natoms, 500 + case)
    om.set_spins(s)
    pm.set_spins(s)
    op, pp = _both_params(oracle, ib, **h)
    col, ncol = pm.colouring(pp)
    if pm.layout == "octant":   # classes of octant blocks: 3 shell-1 classes, or 15 with J'
        assert ncol == (15 if "Jp" in h else 3)
    elif "Jp" not in h:   # the two sublattices
        assert ncol == 2 and np.array_equal(col, np.arange(om.natoms) % 2)
    seed = 0x0C7A + case
    key = oracle.SweepKey(seed=seed, ensemble=0, replica=0, move=move, r=r, philox_rounds=10)
    n_sweeps = 3
    ib.metropolis_mcs(pm, beta, n_sweeps, 0, 0, 0, 0, 0, r if move == 1 else 0.0, seed=seed, p=pp)
    for sw in range(n_sweeps):
        for c in range(ncol):
            om.colour_pass(col, c, sw, beta, op, key)
    diff = np.abs(pm.get_spins(0) - om.spins).max(axis=1)
    # FP32 against FP64: a decision flips only where ln u + beta dE is within rounding of 0,
    # and a flipped site changes its neighbours' later decisions
    assert (diff > 2e-4).sum() <= max(3, om.natoms // 400), int((diff > 2e-4).sum())


def test_octant_pt_accumulators_track_recomputed_energies(oracle, ib, cuda_ok):
    om, pm = _pair(oracle, ib, "BCC", (8, 8, 6), n_replicas=4)
    pm.init_uniform(5)
    op, pp = _both_params(oracle, ib, J=-1.0, Dz=0.5, B=0.2, bulk=True)
    pt = ib.ParallelTempering(pm, 1.0 / ib.temperature_ladder(0.2, 2.0, 4), pp, seed=3, move=ib._lib.MOVE_BALL)
    assert pt.schedule(5)[2] == 5          # the sublattice-class kernel
    pt.run(5, 6)
    e_run, m_run = pt.energies()
    pt.resync()
    e_new, m_new = pt.energies()
    assert np.max(np.abs(e_run - e_new)) < 1e-5 * pm.numAtoms
    assert np.max(np.abs(m_run - m_new)) < 1e-5 * pm.numAtoms
    for r in range(4):
        om.set_spins(pm.get_spins(r))
        assert abs(e_new[r] - om.canonical_energy(op)) < 1e-6 * pm.numAtoms


@pytest.mark.parametrize("kind,dims,shell2", [("HK", (6, 4, 4), False), ("HK", (4, 4, 6), True),
                                              ("HK", (4, 6, 4), False), ("HK", (8, 4, 6), True)])
@pytest.mark.parametrize("move", [0, 1])
def test_octant_engine_equals_one_launch_per_class(oracle, ib, cuda_ok, kind, dims, shell2, move):
    """The persistent octant engine (every sweep of a round in one launch, tasks per packed
    x-plane with bounded dependency waits) against one launch per colour class: spins,
    exchange permutation and swap counts bit-equal after several rounds of PT, accumulators
    within FP32 rounding of each other (the partial sums are grouped differently)."""
    runs = []
    for sweep_kernel in (3, 0):
        om, pm = _pair(oracle, ib, kind, dims, n_replicas=6)
        assert pm.layout == "octant"
        pm.init_uniform(77, 0)
        kw = dict(J=-1.0, Dz=0.4, B=0.15, bulk=False)
        if shell2:
            kw["Jp"] = 0.2
        op, pp = _both_params(oracle, ib, **kw)
        pt = ib.ParallelTempering(pm, 1.0 / ib.temperature_ladder(0.3, 2.5, 6), pp, seed=11, move=move,
                                  r=0.3, sweep_kernel=sweep_kernel)
        assert pt.schedule(4)[2] == (4 if sweep_kernel == 3 else (6 if dims[2] % 4 == 0 else 3))
        pt.run(4, 5)
        e, m = pt.energies()
        runs.append(([pm.get_spins(r) for r in range(6)], pt.permutation(), pt.swap_stats(), e, m, pm.numAtoms))
        pt.close()
    (s0, p0, st0, e0, m0, n), (s1, p1, st1, e1, m1, _) = runs
    for r in range(6):
        np.testing.assert_array_equal(s0[r], s1[r])
    np.testing.assert_array_equal(p0, p1)
    np.testing.assert_array_equal(st0[0], st1[0])
    np.testing.assert_array_equal(st0[1], st1[1])
    np.testing.assert_allclose(e0, e1, rtol=0, atol=1e-6 * n)
    np.testing.assert_allclose(m0, m1, rtol=0, atol=1e-6 * n)


def test_octant_engine_timeout_and_recovery(oracle, ib, cuda_ok):
    """A dependency wait that runs out (the injected stall makes the first class change wait
    for a count nothing reaches) ends the round with ISING_ERR_TIMEOUT after its bound; the
    context stays usable, a resync restores the running energies, and later rounds run
    normally (unit spins, accumulators equal to recomputed energies)."""
    om, pm = _pair(oracle, ib, "HK", (4, 6, 4), n_replicas=4)
    pm.init_uniform(9, 0)
    op, pp = _both_params(oracle, ib, J=-1.0, Dz=0.4, B=0.1, bulk=False)
    pt = ib.ParallelTempering(pm, 1.0 / ib.temperature_ladder(0.3, 2.0, 4), pp, seed=5, move=1, r=0.3,
                              sweep_kernel=3)
    pt.run(2, 1)
    pt.inject_stall(150)
    with pytest.raises(ib.IsingError) as e:
        pt.run(2, 1)
    assert e.value.status == 4
    pt.resync()
    pt.run(2, 3)
    e_run, _ = pt.energies()
    e_dev, _ = ib.observables(pm, pp)
    assert np.max(np.abs(e_run - e_dev)) < 1e-5 * pm.numAtoms
    for r in range(4):
        s = pm.get_spins(r)
        assert np.max(np.abs(np.linalg.norm(s, axis=1) - 1.0)) < 1e-5
    pt.close()


def test_octant_engine_option_errors(oracle, ib, cuda_ok):
    """The persistent octant engine is refused where it cannot run (a checkerboard mesh), and
    the stall hook without the engine or with a bound outside 1..60000 ms is refused."""
    sc = ib.ChainMesh.simple_cubic(8, n_replicas=2)
    pp = ib.params(J=-1.0, Dz=0.3, B=0.1, dmi="bulk", include_Jp=False)
    with pytest.raises(ib.IsingError) as e:
        ib.ParallelTempering(sc, np.array([1.0, 0.5]), pp, seed=1, sweep_kernel=3)
    assert e.value.status == 1
    pt = ib.ParallelTempering(sc, np.array([1.0, 0.5]), pp, seed=1)
    with pytest.raises(ib.IsingError):
        pt.inject_stall(100)
    pt.close()
    om, pm = _pair(oracle, ib, "HK", (4, 4, 4), n_replicas=2)
    op, bp = _both_params(oracle, ib, J=-1.0, Dz=0.3, B=0.1)
    pt = ib.ParallelTempering(pm, np.array([1.0, 0.5]), bp, seed=1, sweep_kernel=3)
    for bad in (0, 60001):
        with pytest.raises(ib.IsingError) as e:
            pt.inject_stall(bad)
        assert e.value.status == 1
    pt.run(2, 1)
    pt.close()


FCC = (np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]], np.float32), (1.0, 1.0, 1.0, 90.0, 90.0, 90.0))


@pytest.mark.parametrize("Jp,ncol,dims", [(0.0, 4, (4, 4, 8)), (0.2, 10, (6, 4, 4)), (0.2, 10, (4, 4, 6))])
def test_fcc_block_classes_replay_the_oracle(oracle, ib, cuda_ok, Jp, ncol, dims):
    """A cell that is not one of the reference's (FCC, 4 sublattices) on the octant layout:
    without J' its sublattices are the classes, with J' 10 DSatur classes of whole blocks, on
    the pair kernel (nz % 4 == 0) and the one-site kernel; sweeps replay the oracle's colour
    passes as for the reference cells."""
    frac, (a, b, c, ab, bc, ca) = FCC
    om = oracle.Mesh(frac, *dims, a, b, c, ab, bc, ca)
    pm = ib.ChainMesh(*dims, frac, a, b, c, ab, bc, ca)
    assert pm.layout == "octant"
    s = _random_spins(om.natoms, 77)
    om.set_spins(s)
    pm.set_spins(s)
    op, pp = _both_params(oracle, ib, J=-1.0, Jp=Jp, Dz=0.3, B=0.1, bulk=False)
    col, n = pm.colouring(pp)
    assert n == ncol
    seed, r, beta = 0xFCC, 0.25, 1.2
    key = oracle.SweepKey(seed=seed, ensemble=0, replica=0, move=1, r=r, philox_rounds=10)
    ib.metropolis_mcs(pm, beta, 3, 0, 0, 0, 0, 0, r, seed=seed, p=pp)
    for sw in range(3):
        for k in range(n):
            om.colour_pass(col, k, sw, beta, op, key)
    diff = np.abs(pm.get_spins(0) - om.spins).max(axis=1)
    assert (diff > 2e-4).sum() <= max(3, om.natoms // 400), int((diff > 2e-4).sum())
