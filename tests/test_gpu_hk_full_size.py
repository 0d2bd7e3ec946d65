"""Hyper-kagome (the crystal of src/ISING.f90:105) on its block classes at the bench size,
48^3 cells x 16 replicas = 21,233,664 sites, without J' (3 shell-1 classes) and with J' (15
classes of a DSatur colouring), through the PT object: size-independent properties after 3
rounds of 10 sweeps -- the running FP64 accumulators equal the recomputed energies and
magnetisations, every spin stays a unit vector, and the schedule is the pair kernel with the
expected launches.  At 24^3 x 4 the recomputed energy of every replica also equals the FP64
oracle's canonical energy of the downloaded spins."""
import numpy as np
import pytest

from test_gpu_parity import _both_params

pytestmark = pytest.mark.gpu


def _hk(ib, n, reps):
    a, b, c, ab, bc, ca, f = ib.hyper_kagome_unit_cell()
    return ib.ChainMesh(n, n, n, f, a, b, c, ab, bc, ca, n_replicas=reps)


@pytest.mark.parametrize("Jp,classes", [(0.0, 3), (0.1, 15)])
def test_hk_bench_size_accumulators_and_norms(ib, cuda_ok, Jp, classes):
    pm = _hk(ib, 48, 16)
    assert pm.layout == "octant"
    pm.init_uniform(0x15196)
    pp = ib.params(J=-1.0, J_prime=Jp, Dz=0.3, B=0.1, dmi="interfacial")
    pt = ib.ParallelTempering(pm, 1.0 / ib.temperature_ladder(0.1, 2.0, 16), pp, seed=7, move=ib._lib.MOVE_BALL,
                              r=0.2)
    group, launches, kernel = pt.schedule(10)
    assert kernel == 6 and launches == 10 * classes
    pt.run(10, 3)
    e_run, m_run = pt.energies()
    pt.resync()
    e_new, m_new = pt.energies()
    n = pm.numAtoms
    assert np.max(np.abs(e_run - e_new)) < 1e-6 * n
    assert np.max(np.abs(m_run - m_new)) < 1e-6 * n
    for r in (0, 7, 15):
        s = pm.get_spins(r)
        assert np.max(np.abs(np.linalg.norm(s, axis=1) - 1.0)) < 2e-6
    pt.close()


def test_hk_energies_equal_the_oracle_after_sweeps(oracle, ib, cuda_ok):
    frac, (a, b, c, ab, bc, ca) = oracle.HYPER_KAGOME_CELL
    om = oracle.Mesh(frac, 24, 24, 24, a, b, c, ab, bc, ca)
    pm = _hk(ib, 24, 4)
    pm.init_uniform(11)
    op, pp = _both_params(oracle, ib, J=-1.0, Jp=0.1, Dz=0.3, B=0.1, bulk=False)
    pt = ib.ParallelTempering(pm, 1.0 / ib.temperature_ladder(0.2, 2.0, 4), pp, seed=3, move=ib._lib.MOVE_BALL,
                              r=0.2)
    pt.run(5, 4)
    pt.resync()
    e_dev, _ = pt.energies()
    for r in range(4):
        om.set_spins(pm.get_spins(r))
        assert abs(e_dev[r] - om.canonical_energy(op)) < 1e-6 * pm.numAtoms
    pt.close()
