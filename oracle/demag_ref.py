"""Test infrastructure: FP64 numpy restatement of the reference's demagnetising field, the
checker of the library's device implementation (never called by the product).

Follows src/reciprocalSpaceProcesses.f90 (rsp):
- interpolate_to_fft_array (rsp:76-126): cloud-in-cell deposit of the spins onto one grid
  point per mesh cell (the cell centre, src/chainMesh.f90:862-867); a cell gathers the atoms of
  its 27 neighbouring cells (src/chainMesh.f90:85-131) with weight
  prod_i max(1 - |d_i|, 0), d the atom's offset from the centre in units of the Bravais
  vectors, minimum image (distance_points_vec_bravais, src/chainMesh.f90:244-276), atom
  positions as the single-precision values makeChainMesh stores (src/chainMesh.f90:868-877);
- fft_forward_chainMesh (rsp:178-185): real-to-complex 3-D transforms of the three
  components, the first (x) index halved;
- calculate_demagnetisation_field (rsp:202-281): H(k) = -(k.M / k^2) k with
  k = 2 pi (wx/N) ar + 2 pi (wy/L) br + 2 pi (wz/M) cr (wy, wz folded to the signed range,
  wx in 0..N/2), the k = 0 bin zero, and every bin with |k_x| > pi/a, |k_y| > pi/b or
  |k_z| > pi/c set to zero (a, b, c the lattice constants as given); backward complex-to-real transforms divided by N L M;
- interpolate_fft_to_atoms (rsp:128-176): the same weights carry the grid field back to the
  atoms.
The constant pi is the reference's default-real literal (src/constants.f90), i.e. pi rounded
to single precision; the energies use mu_0 = 1.25663706127e-6 (src/constants.f90:15).

FFTW is not in this image, so numpy's FFT stands in for the reference's FFTW plans; the
backward transform of the k-space field (which is not Hermitian in the Nyquist planes of the
unhalved axes, where the folded wave index stays positive) is numpy's irfftn: complex inverse
transforms along y and z, then the real inverse along x.
"""
from __future__ import annotations

import numpy as np

PI_F = float(np.float32(3.14159265358979323846))
MU_0 = 1.25663706127e-6


def cic_pairs(mesh):
    """(cell index [P], atom index [P], weight [P]) of every (cell, atom) pair with a non-zero
    weight; cells in reference order (ix * ny + iy) * nz + iz."""
    nx, ny, nz, nsub = mesh.nx, mesh.ny, mesh.nz, mesh.nsub
    v = mesh.vectors()
    av, bv, cv, ar, br, cr = v
    pos = mesh.positions().astype(np.float64)                 # real(4) positions, widened
    natoms = pos.shape[0]
    atoms = np.arange(natoms)
    acell = atoms // nsub
    aix, rem = np.divmod(acell, ny * nz)
    aiy, aiz = np.divmod(rem, nz)
    cells, ats, ws = [], [], []
    for ox in (-1, 0, 1):
        for oy in (-1, 0, 1):
            for oz in (-1, 0, 1):
                # the cell whose 27-neighbourhood contains the atom's cell at offset (ox, oy, oz)
                cx, cy, cz = (aix - ox) % nx, (aiy - oy) % ny, (aiz - oz) % nz
                centre = (np.outer(cx + 0.5, av) + np.outer(cy + 0.5, bv) + np.outer(cz + 0.5, cv))
                d = pos - centre
                a_c = d @ ar
                b_c = d @ br
                c_c = d @ cr
                a_c = a_c - nx * np.rint(a_c / nx)
                b_c = b_c - ny * np.rint(b_c / ny)
                c_c = c_c - nz * np.rint(c_c / nz)
                w = (np.maximum(1.0 - np.abs(a_c), 0.0) * np.maximum(1.0 - np.abs(b_c), 0.0)
                     * np.maximum(1.0 - np.abs(c_c), 0.0))
                keep = w != 0.0
                cells.append(((cx * ny + cy) * nz + cz)[keep])
                ats.append(atoms[keep])
                ws.append(w[keep])
    return np.concatenate(cells), np.concatenate(ats), np.concatenate(ws)


def demag_field(mesh, spins):
    """H per atom [natoms, 3] of spins [natoms, 3] (calculate_demagnetisation_field)."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    # the cut-off takes the lattice constants as given (chainMesh%a, %b, %c,
    # src/chainMesh.f90:792-794), not the lengths of the Bravais vectors, which differ in the
    # last bits (sin of the single-precision right angle is not 1); on a Nyquist plane
    # |k_i| equals pi/a_i to rounding, so the choice decides whether that plane is cut
    a, b, c = mesh.a, mesh.b, mesh.c
    ar, br, cr = mesh.vectors()[3:]
    cell, atom, w = cic_pairs(mesh)
    ncell = nx * ny * nz
    grid = np.zeros((3, ncell))
    for q in range(3):
        np.add.at(grid[q], cell, w * spins[atom, q])
    G = grid.reshape(3, nx, ny, nz)
    F = np.stack([np.fft.rfftn(G[q], axes=(1, 2, 0)) for q in range(3)])   # [3, nx/2+1, ny, nz]
    wx = np.arange(nx // 2 + 1, dtype=np.float64)
    wy = np.arange(ny)
    wy = np.where(wy > ny // 2, wy - ny, wy).astype(np.float64)
    wz = np.arange(nz)
    wz = np.where(wz > nz // 2, wz - nz, wz).astype(np.float64)
    kx = (2 * PI_F * (wx / nx))[:, None] * ar[None, :]
    ky = (2 * PI_F * (wy / ny))[:, None] * br[None, :]
    kz = (2 * PI_F * (wz / nz))[:, None] * cr[None, :]
    K = kx[:, None, None, :] + ky[None, :, None, :] + kz[None, None, :, :]   # [i, j, k, 3]
    k2 = (K * K).sum(-1)
    kdm = K[..., 0] * F[0] + K[..., 1] * F[1] + K[..., 2] * F[2]
    with np.errstate(invalid="ignore", divide="ignore"):
        Hk = np.stack([-(kdm / k2) * K[..., q] for q in range(3)])
    cut = (np.abs(K[..., 0]) > PI_F / a) | (np.abs(K[..., 1]) > PI_F / b) | (np.abs(K[..., 2]) > PI_F / c)
    Hk[:, cut] = 0.0
    Hk[:, 0, 0, 0] = 0.0
    Hg = np.stack([np.fft.irfftn(Hk[q], s=(ny, nz, nx), axes=(1, 2, 0)) for q in range(3)])
    Hg = Hg.reshape(3, ncell)                       # irfftn already divides by N L M
    H = np.zeros((spins.shape[0], 3))
    for q in range(3):
        np.add.at(H[:, q], atom, w * Hg[q][cell])
    return H


def demag_energy(spins, H):
    """-1/2 mu_0 sum_i S_i . H_i: the demagnetising part of TotalHeisenbergEnergy
    (calculateTotalHeisenbergEnergyHelper, src/energyMin.f90:223-226)."""
    return -0.5 * MU_0 * float((spins * H).sum())
