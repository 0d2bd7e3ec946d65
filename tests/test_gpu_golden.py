"""The CUDA path against the committed golden fixtures (tests/golden, made by the oracle).
Tolerances as in test_gpu_parity: 1e-6 of the per-site energy scale, 1e-9 per winding slice."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
HAM = dict(J=-1.0, J_prime=0.15, Dz=0.4, B=0.2, K=0.05, K_axis=(0.0, 0.6, 0.8))
CELLS = {"sc4": ("SC", (4, 4, 4)), "sc6": ("SC", (6, 6, 6)), "sc8": ("SC", (8, 8, 8)), "sc16": ("SC", (16, 16, 16)),
         "bcc3": ("BCC", (3, 3, 3)), "hk3": ("HK", (3, 3, 3))}


@pytest.mark.parametrize("name", sorted(CELLS))
def test_gpu_matches_fixture(ib, cuda_ok, name):
    kind, dims = CELLS[name]
    g = np.load(os.path.join(GOLD, f"{name}.npz"))
    cell = {"SC": ib.sc_unit_cell, "BCC": ib.bcc_unit_cell, "HK": ib.hyper_kagome_unit_cell}[kind]()
    a, b, c, ab, bc, ca, frac = cell
    if kind == "SC":
        a = b = c = 1.0
    m = ib.ChainMesh(*dims, frac, a, b, c, ab, bc, ca, n_replicas=2)
    m.init_uniform(0x15196, ensemble=3)
    assert np.allclose(m.get_spins(1), g["init"], atol=2e-6)
    m.set_spins(g["spins0"], 0)
    z1 = len(m.neighbours(0, 0))
    z2 = len(m.neighbours(0, 1))
    scale = 1.0 * z1 + 0.4 * z1 + 0.15 * z2 + 0.2 + 0.05
    for bulk in (0, 1):
        p = ib.params(dmi="bulk" if bulk else "interfacial", **HAM)
        old, new = ib.local_energy_batch(m, g["atoms"], g["prop"], p, replica=0)
        assert np.allclose(old, g[f"local_b{bulk}"][:, 0], rtol=0, atol=1e-6 * scale)
        assert np.allclose(new, g[f"local_b{bulk}"][:, 1], rtol=0, atol=1e-6 * scale)
        e, _ = ib.observables(m, p)
        assert abs(e[0] - float(g[f"canonical_b{bulk}"])) <= 1e-6 * m.numAtoms * scale
        pt_ = ib.reference_params("total", HAM["J"], 0.0, HAM["Dz"], 0.0, HAM["B"])
        pt_.dmi_mode = bulk
        pt_.K = HAM["K"]
        pt_.K_axis[:] = list(HAM["K_axis"])
        et = ib.total_heisenberg_energy(m, 0, 0, 0, 0, 0, p=pt_)
        assert abs(et - float(g[f"total_ref_b{bulk}"])) <= 1e-6 * m.numAtoms * scale
    q = ib.winding_all_slices(m, 0)
    assert np.allclose(q, g["q_slices"], atol=1e-9)
    assert [round(v) for v in q] == [round(v) for v in g["q_slices"]]
    wm, ws, mag = ib.chain_mesh_statistics(m, 0)
    assert np.allclose([wm, ws, *mag], g["stats"], atol=1e-9)
    if "sweep_spins" in g.files:
        p = ib.params(dmi="bulk", **{k: v for k, v in HAM.items() if k != "J_prime"})
        ib.metropolis_mcs(m, 1.5, 1, 0, 0, 0, 0, 0, 0.2, seed=0xABCDEF, p=p, replica=0)
        d = np.abs(m.get_spins(0) - g["sweep_spins"]).max(axis=1)
        assert (d > 2e-5).sum() <= 2, (d > 2e-5).sum()
    m.close()
