"""Known answers of the oracle's restatement of calculate_demagnetisation_field
(src/reciprocalSpaceProcesses.f90:76-281, oracle/demag_ref.py): a uniform magnetisation has no
demagnetising field (only the removed k = 0 bin); a helix whose spins rotate in the plane
normal to its wave vector is divergence-free (k.M = 0), so its field vanishes; a longitudinal
spiral M = (cos qx, sin qx, 0) has H = -c M_x x_hat with one factor c in (0, 1] at every atom
(the cloud-in-cell smoothing of one Fourier mode) and no y or z component; the cloud-in-cell
weights of an atom sum to 1 when its cell's 27-neighbourhood holds all its weight."""
import numpy as np


def _sc(oracle, L):
    return oracle.Mesh.sc(L)


def test_uniform_and_divergence_free_fields_vanish(oracle):
    from oracle import demag_ref as D
    m = _sc(oracle, 8)
    n = m.natoms
    s = np.tile([0.3, -0.4, np.sqrt(1 - 0.25)], (n, 1))
    assert np.abs(D.demag_field(m, s)).max() < 1e-12
    z = m.positions()[:, 2].astype(np.float64)
    q = 2 * np.pi / 8
    helix = np.stack([np.cos(q * z), np.sin(q * z), np.zeros(n)], 1)
    assert np.abs(D.demag_field(m, helix)).max() < 1e-12


def test_longitudinal_spiral_field(oracle):
    from oracle import demag_ref as D
    m = _sc(oracle, 8)
    n = m.natoms
    x = m.positions()[:, 0].astype(np.float64)
    q = 2 * np.pi / 8
    s = np.stack([np.cos(q * x), np.sin(q * x), np.zeros(n)], 1)
    H = D.demag_field(m, s)
    assert np.abs(H[:, 1:]).max() < 1e-12
    big = np.abs(s[:, 0]) > 0.5
    c = -H[big, 0] / s[big, 0]
    assert 0.0 < c.mean() <= 1.0 and np.ptp(c) < 1e-12


def test_cic_weights_partition_unity(oracle):
    from oracle import demag_ref as D
    for frac, (a, b, c, ab, bc, ca) in (oracle.SC_CELL, oracle.BCC_CELL):
        m = oracle.Mesh(frac, 4, 5, 6, a, b, c, ab, bc, ca)
        _, atom, w = D.cic_pairs(m)
        tot = np.bincount(atom, w, minlength=m.natoms)
        assert np.allclose(tot, 1.0, atol=1e-12)
