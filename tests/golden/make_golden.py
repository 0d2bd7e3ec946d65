"""Regenerate the golden fixtures of tests/golden from the CPU oracle.

The reference ships no golden vectors for this path and cannot be built here, so these
fixtures pin the oracle (and, in the GPU tests, the CUDA path) to fixed seeded cases:
spins from the Philox initialiser, per-site energies for fixed proposals, total energies in
both routine conventions, per-slice winding numbers and one colour-class sweep.

Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402

CASES = {
    "sc4": (O.SC_CELL, (4, 4, 4)),
    "sc6": (O.SC_CELL, (6, 6, 6)),
    "sc8": (O.SC_CELL, (8, 8, 8)),
    "sc16": (O.SC_CELL, (16, 16, 16)),
    "bcc3": (O.BCC_CELL, (3, 3, 3)),
    "hk3": (O.HYPER_KAGOME_CELL, (3, 3, 3)),
}
HAM = dict(J=-1.0, J_prime=0.15, Dz=0.4, B=0.2, K=0.05, K_axis=(0.0, 0.6, 0.8))


def make(name):
    (frac, (a, b, c, ab, bc, ca)), dims = CASES[name]
    m = O.Mesh(frac, *dims, a, b, c, ab, bc, ca)
    m.init_uniform(0x15196, 3, 1)
    init = m.spins.copy()
    # FP32-representable spins, so the FP32 device state holds exactly the same configuration
    m.set_spins(init.astype(np.float32).astype(np.float64))
    spins0 = m.spins.copy()
    rng = np.random.default_rng(2024)
    atoms = rng.choice(m.natoms, size=min(64, m.natoms), replace=False).astype(np.int64)
    prop = rng.normal(size=(len(atoms), 3))
    prop /= np.linalg.norm(prop, axis=1, keepdims=True)
    out = {"init": init, "spins0": spins0, "atoms": atoms, "prop": prop.astype(np.float32).astype(np.float64)}
    prop = out["prop"]
    for bulk in (0, 1):
        p = O.Params(dmi_bulk=bool(bulk), **HAM)
        le = np.array([m.local_energy(int(a_), p, prop[k]) for k, a_ in enumerate(atoms)])
        out[f"local_b{bulk}"] = le
        out[f"total_ref_b{bulk}"] = np.array(m.total_energy(p, 2.0))
        out[f"canonical_b{bulk}"] = np.array(m.canonical_energy(p))
    out["q_slices"] = np.array([m.winding_number(z) for z in range(1, dims[2] + 1)])
    wm, ws, mag = m.statistics()
    out["stats"] = np.array([wm, ws, *mag])
    # one checkerboard sweep (both colour classes) of the simple cubic cases
    if name.startswith("sc") and dims[2] % 4 == 0:
        col = O.checkerboard(*dims)
        p = O.Params(dmi_bulk=True, **{k: v for k, v in HAM.items() if k != "J_prime"})
        key = O.SweepKey(seed=0xABCDEF, ensemble=0, replica=0, move=1, r=0.2, philox_rounds=10)
        n0, de0 = m.colour_pass(col, 0, 0, 1.5, p, key)
        n1, de1 = m.colour_pass(col, 1, 0, 1.5, p, key)
        out["sweep_spins"] = m.spins.copy()
        out["sweep_de"] = np.array(de0 + de1)
        out["sweep_acc"] = np.array(n0 + n1)
    return out


def main():
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **make(name))
        print("wrote", name)


if __name__ == "__main__":
    main()
