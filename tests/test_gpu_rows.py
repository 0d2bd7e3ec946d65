"""GPU parity of the row-per-warp checkerboard kernel (nz = 64 or 128) and of the paired
L2 schedule (second colour of replica group g-1 with the first colour of group g) against
the oracle's colour passes with the same Philox keys."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _spins(n, seed):
    rng = np.random.default_rng(seed)
    s = rng.normal(size=(n, 3))
    s /= np.linalg.norm(s, axis=1, keepdims=True)
    return s.astype(np.float32).astype(np.float64)


CASES = [((4, 6, 128), dict(J=-1.0, Dz=0.7, B=0.3, K=0.05, bulk=True), 1, 0.2, 3.0),
         ((6, 4, 64), dict(J=-1.0, Dz=0.5, B=0.2, bulk=True), 0, 0.0, 1.0),
         ((4, 4, 128), dict(J=1.0, Dz=0.4, B=-0.1, bulk=False), 1, 0.3, 2.0),
         ((4, 4, 64), dict(J=-1.0, Dz=0.0, B=0.25, K=0.1, bulk=False), 0, 0.0, 0.7)]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_rows_kernel_replay(oracle, ib, cuda_ok, case):
    dims, h, move, r, beta = CASES[case]
    om = oracle.Mesh(oracle.SC_CELL[0], *dims, 1.0, 1.0, 1.0)
    pm = ib.ChainMesh(*dims, oracle.SC_CELL[0], 1.0, 1.0, 1.0)
    assert pm.checkerboard
    s = _spins(om.natoms, 70 + case)
    om.set_spins(s)
    pm.set_spins(s)
    op = oracle.Params(J=h["J"], Dz=h["Dz"], B=h["B"], K=h.get("K", 0.0), dmi_bulk=h["bulk"])
    pp = ib.params(J=h["J"], Dz=h["Dz"], B=h["B"], K=h.get("K", 0.0), dmi="bulk" if h["bulk"] else "interfacial")
    seed = 0xC0FFEE + case
    n_sw = 3
    ib.metropolis_mcs(pm, beta, n_sw, 0, 0, 0, 0, 0, r if move else 0.0, seed=seed, p=pp)
    col = oracle.checkerboard(*dims)
    key = oracle.SweepKey(seed=seed, ensemble=0, replica=0, move=move, r=r, philox_rounds=10)
    for sw in range(n_sw):
        om.colour_pass(col, 0, sw, beta, op, key)
        om.colour_pass(col, 1, sw, beta, op, key)
    diff = np.abs(pm.get_spins(0) - om.spins).max(axis=1)
    assert (diff > 2e-5).sum() <= 2, ((diff > 2e-5).sum(), diff.max())


@pytest.mark.parametrize("group", [1, 2, 3])
def test_paired_schedule_replay(oracle, ib, cuda_ok, group):
    dims = (4, 6, 128)
    R = 5
    om = oracle.Mesh(oracle.SC_CELL[0], *dims, 1.0, 1.0, 1.0)
    pm = ib.ChainMesh(*dims, oracle.SC_CELL[0], 1.0, 1.0, 1.0, n_replicas=R)
    init = [_spins(om.natoms, 100 + rr) for rr in range(R)]
    for rr in range(R):
        pm.set_spins(init[rr], rr)
    op = oracle.Params(J=-1.0, Dz=0.5, B=0.2, K=0.05, dmi_bulk=True)
    pp = ib.params(J=-1.0, Dz=0.5, B=0.2, K=0.05, dmi="bulk")
    betas = 1.0 / ib.temperature_ladder(0.3, 2.0, R)
    k = 3
    pt = ib.ParallelTempering(pm, betas, pp, seed=99, ensemble=2, move=ib._lib.MOVE_BALL, r=0.2,
                              l2_group=group)
    pt.run(k, 1)
    e_run, m_run = pt.energies()
    col = oracle.checkerboard(*dims)
    for rr in range(R):
        om.set_spins(init[rr])
        key = oracle.SweepKey(seed=99, ensemble=2, replica=rr, move=1, r=0.2, philox_rounds=10)
        for sw in range(k):
            om.colour_pass(col, 0, sw, betas[rr], op, key)
            om.colour_pass(col, 1, sw, betas[rr], op, key)
        g = pm.get_spins(rr)
        diff = np.abs(g - om.spins).max(axis=1)
        assert (diff > 2e-5).sum() <= 2, (rr, (diff > 2e-5).sum())
        # running FP64 energy of the replica vs the oracle on the GPU's final spins
        om.set_spins(g)
        assert abs(e_run[rr] - om.canonical_energy(op)) <= 2e-6 * om.natoms * 9
    pt.close()


@pytest.mark.parametrize("dims", [(4, 6, 128), (6, 4, 64), (8, 8, 8), (10, 12, 16)])
def test_tma_and_register_kernels_agree(ib, cuda_ok, dims):
    """The TMA-staged and the register colour pass make the same decisions (same keys)."""
    R = 3
    outs = []
    for kern in (1, 2):
        pm = ib.ChainMesh(*dims, np.zeros((1, 3), np.float32), 1.0, 1.0, 1.0, n_replicas=R)
        for rr in range(R):
            pm.set_spins(_spins(pm.numAtoms, 300 + rr), rr)
        pp = ib.params(J=-1.0, Dz=0.6, B=0.2, K=0.03, dmi="bulk")
        pt = ib.ParallelTempering(pm, 1.0 / ib.temperature_ladder(0.5, 2.0, R), pp, seed=5, move=ib._lib.MOVE_BALL,
                                  r=0.25, l2_group=1, sweep_kernel=kern)
        pt.run(4, 2)
        outs.append([pm.get_spins(rr) for rr in range(R)] + [pt.energies()[0]])
        pt.close()
    for rr in range(R):
        d = np.abs(outs[0][rr] - outs[1][rr]).max(axis=1)
        assert (d > 2e-5).sum() <= 2, (rr, (d > 2e-5).sum())
    assert np.allclose(outs[0][R], outs[1][R], rtol=1e-6, atol=1e-3)
